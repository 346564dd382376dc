// The learned denoiser: a kernel-predicting U-Net run and trained on the
// device by the BF16 tensor-core kernels of nn.cu.
//
// Five levels of 32, 64, 96, 128 and 160 channels, two 3x3 convolutions
// (bias, ReLU) per level on the way down and on the way up, 2x2 average
// pooling down, nearest 2x upsampling up, skip connections concatenated
// ahead of the upsampled channels, and a 3x3 head of 32 fp32 outputs: 25
// logits of a 5 x 5 per-pixel filter and one log relative-error estimate.
// The filter is applied to the demodulated radiance (k_kpn).
//
// Every activation is NHWC bf16. An encoder level's second convolution
// writes straight into the tail channels of the decoder's concatenation
// buffer at that level, and the upsampling writes its head channels, so the
// concatenation costs no copy; the matching gradient buffers work the same
// way (pooling's gradient is added into the skip channels the decoder's
// data gradient already wrote).
//
// phiray has no learned denoiser (its Denoise is the a-trous filter of
// src/kernel/denoise.wgsl); the per-tile fallback to that filter keeps its
// behaviour wherever the network's own error estimate is high.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace phx {
namespace {

constexpr int NL = 19;
// Layer order: e0a e0b e1a e1b e2a e2b e3a e3b ba bb d3a d3b d2a d2b d1a d1b d0a d0b head.
constexpr int CIN[NL] = {16, 32, 32, 64, 64, 96, 96, 128, 128, 160, 288, 128, 224, 96, 160, 64, 96, 32, 32};
constexpr int COUT[NL] = {32, 32, 64, 64, 96, 96, 128, 128, 160, 160, 128, 128, 96, 96, 64, 64, 32, 32, 32};
constexpr int LEVEL_CH[5] = {32, 64, 96, 128, 160};
constexpr int CAT_CH[4] = {96, 160, 224, 288};  // up channels + skip channels
constexpr int UP_CH[4] = {64, 96, 128, 160};    // offset of the skip channels
constexpr int FEAT = 16;
constexpr int HEAD = 32;

int round64(int k) { return (k + 63) / 64 * 64; }

struct Conv {
    int cin = 0, cout = 0, K = 0, Kp = 0, Kp2 = 0;
    DevMem w32, wb, b32, mw, vw, mb, vb, w2;
    float* gw = nullptr;  // weight gradient [Kp][cout], in the network's gradient arena
    float* gb = nullptr;  // bias gradient [cout], in the arena
};

// Offsets (in floats, each a multiple of 64) of every layer's weight and bias
// gradients in one arena, so a data-parallel trainer reduces all gradients
// with one collective; the arena's total length in floats.
size_t grad_layout(size_t* off_w, size_t* off_b) {
    size_t at = 0;
    for (int i = 0; i < NL; i++) {
        const size_t w = (size_t)COUT[i] * (size_t)((9 * CIN[i] + 63) / 64 * 64);
        if (off_w) off_w[i] = at;
        at += (w + 63) / 64 * 64;
        if (off_b) off_b[i] = at;
        at += ((size_t)COUT[i] + 63) / 64 * 64;
    }
    return at;
}

// A bf16 NHWC view: base, pixel pitch, channel offset.
struct View {
    void* p;
    int pitch, off;
};

struct Shape {
    int B = 0, H = 0, W = 0;
    bool train = false;
    bool operator==(const Shape& o) const { return B == o.B && H == o.H && W == o.W && train == o.train; }
};

}  // namespace
}  // namespace phx

struct phx_unet_s {
    phx_ctx handle = nullptr;
    phx::Ctx* ctx = nullptr;
    phx::Conv L[phx::NL];
    phx::DevMem grads;  // every layer's weight and bias gradients (grad_layout)
    phx::DevMem zero_bias;
    phx::Shape shape;
    // activations
    phx::DevMem A[5], cat[4], pool[5], B4, Da[4], Db[4], logits;
    // gradients
    phx::DevMem dA[5], dcat[4], dpool[5], dB4, dDa[4], dDb[4], dlogits;
    // tracer-facing scratch
    phx::DevMem feat, irr, irr_clamped, alb, out, err, tile_err, fallback;
    phx::DevMem ffeat, firr, falb, fout, ferr;  // the mirrored inputs and outputs of the flip average
    bool clamp = false;  // firefly clamp on the irradiance the predicted kernels filter
    int flips = 1;       // images the result is averaged over: 1, 2 (+ mirrored in x) or 4 (+ in y, both)
    int step = 0;
    float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
};

namespace phx {
namespace {

size_t level_px(const Shape& s, int l) { return (size_t)s.B * (s.H >> l) * (s.W >> l); }

int32_t ensure(phx_unet_s* n, const Shape& s) {
    if (n->shape == s) return PHX_OK;
    const size_t bf = sizeof(__nv_bfloat16);
    for (int l = 0; l < 5; l++) {
        const size_t P = level_px(s, l);
        PHX_TRY(n->A[l].reserve(P * LEVEL_CH[l] * bf));
        if (l > 0) PHX_TRY(n->pool[l].reserve(P * LEVEL_CH[l - 1] * bf));
        if (l < 4) {
            PHX_TRY(n->cat[l].reserve(P * CAT_CH[l] * bf));
            PHX_TRY(n->Da[l].reserve(P * LEVEL_CH[l] * bf));
            PHX_TRY(n->Db[l].reserve(P * LEVEL_CH[l] * bf));
        }
        if (s.train) {
            PHX_TRY(n->dA[l].reserve(P * LEVEL_CH[l] * bf));
            if (l > 0) PHX_TRY(n->dpool[l].reserve(P * LEVEL_CH[l - 1] * bf));
            if (l < 4) {
                PHX_TRY(n->dcat[l].reserve(P * CAT_CH[l] * bf));
                PHX_TRY(n->dDa[l].reserve(P * LEVEL_CH[l] * bf));
                PHX_TRY(n->dDb[l].reserve(P * LEVEL_CH[l] * bf));
            }
        }
    }
    const size_t P4 = level_px(s, 4), P0 = level_px(s, 0);
    PHX_TRY(n->B4.reserve(P4 * 160 * bf));
    PHX_TRY(n->logits.reserve(P0 * HEAD * sizeof(float)));
    if (s.train) {
        PHX_TRY(n->dB4.reserve(P4 * 160 * bf));
        PHX_TRY(n->dlogits.reserve(P0 * HEAD * bf));
    }
    n->shape = s;
    return PHX_OK;
}

// One 3x3 convolution of `in` (cin channels) by weights `w` ([cout][Kp] bf16),
// output channels tiled into launches of at most 160.
int32_t conv(phx_unet_s* n, View in, int cin, const void* w, int Kp, const float* bias, View out, int cout,
             const Shape& s, int level, bool relu, bool f32) {
    const int H = s.H >> level, W = s.W >> level;
    int n0 = 0;
    while (n0 < cout) {
        const int left = cout - n0;
        const int t = left >= 160 ? 160 : (left >= 128 ? 128 : (left >= 96 ? 96 : (left >= 64 ? 64 : 32)));
        const char* wt = (const char*)w + (size_t)n0 * Kp * sizeof(__nv_bfloat16);
        PHX_TRY(phx_nn_conv_fwd(n->handle, in.p, in.pitch, in.off, cin, wt, Kp, bias + n0, out.p, out.pitch,
                                out.off + n0, t, s.B, H, W, relu ? 1 : 0, f32 ? 1 : 0));
        n0 += t;
    }
    return PHX_OK;
}

int32_t layer_fwd(phx_unet_s* n, int i, View in, View out, const Shape& s, int level) {
    Conv& c = n->L[i];
    const bool head = i == NL - 1;
    return conv(n, in, c.cin, c.wb.ptr, c.Kp, (const float*)c.b32.ptr, out, c.cout, s, level, !head, head);
}

// Backward of layer i: dy (its output gradient, ReLU already applied),
// x (its input), dx (nullable: the input gradient, written).
int32_t layer_bwd(phx_unet_s* n, int i, View x, View dy, View* dx, const Shape& s, int level) {
    Conv& c = n->L[i];
    const int H = s.H >> level, W = s.W >> level;
    PHX_TRY(phx_nn_conv_wgrad(n->handle, x.p, x.pitch, x.off, c.cin, dy.p, dy.pitch, dy.off, c.cout,
                              c.gw, c.Kp, s.B, H, W));
    PHX_TRY(phx_nn_bias_grad(n->handle, dy.p, dy.pitch, dy.off, c.cout, s.B * H * W, c.gb));
    if (dx)
        PHX_TRY(conv(n, dy, c.cout, c.w2.ptr, c.Kp2, (const float*)n->zero_bias.ptr, *dx, c.cin, s, level, false,
                     false));
    return PHX_OK;
}

int32_t relu_bwd(phx_unet_s* n, View y, View dy, int C, const Shape& s, int level) {
    return phx_nn_relu_bwd(n->handle, y.p, y.pitch, y.off, dy.p, dy.pitch, dy.off, C, (int)level_px(s, level));
}

View v(DevMem& m, int pitch, int off = 0) { return View{m.ptr, pitch, off}; }

// Every layer up to the head's input (Db[0]); with_head: the head too (fp32 logits).
int32_t forward(phx_unet_s* n, const void* feat, const Shape& s, bool with_head = true) {
    View x{(void*)feat, FEAT, 0};
    for (int l = 0; l < 4; l++) {
        PHX_TRY(layer_fwd(n, 2 * l, x, v(n->A[l], LEVEL_CH[l]), s, l));
        PHX_TRY(layer_fwd(n, 2 * l + 1, v(n->A[l], LEVEL_CH[l]), v(n->cat[l], CAT_CH[l], UP_CH[l]), s, l));
        PHX_TRY(phx_nn_pool_fwd(n->handle, n->cat[l].ptr, CAT_CH[l], UP_CH[l], LEVEL_CH[l], s.B, s.H >> l, s.W >> l,
                                n->pool[l + 1].ptr));
        x = v(n->pool[l + 1], LEVEL_CH[l]);
    }
    PHX_TRY(layer_fwd(n, 8, x, v(n->A[4], 160), s, 4));
    PHX_TRY(layer_fwd(n, 9, v(n->A[4], 160), v(n->B4, 160), s, 4));
    View below = v(n->B4, 160);
    int below_ch = 160;
    for (int l = 3; l >= 0; l--) {
        PHX_TRY(phx_nn_up_fwd(n->handle, below.p, below_ch, s.B, s.H >> l, s.W >> l, n->cat[l].ptr, CAT_CH[l], 0));
        const int d = 10 + 2 * (3 - l);
        PHX_TRY(layer_fwd(n, d, v(n->cat[l], CAT_CH[l]), v(n->Da[l], LEVEL_CH[l]), s, l));
        PHX_TRY(layer_fwd(n, d + 1, v(n->Da[l], LEVEL_CH[l]), v(n->Db[l], LEVEL_CH[l]), s, l));
        below = v(n->Db[l], LEVEL_CH[l]);
        below_ch = LEVEL_CH[l];
    }
    if (!with_head) return PHX_OK;
    return layer_fwd(n, 18, below, View{n->logits.ptr, HEAD, 0}, s, 0);
}

int32_t backward(phx_unet_s* n, const void* feat, const Shape& s) {
    cudaStream_t st = n->ctx->stream;
    PHX_CUDA(cudaMemsetAsync(n->grads.ptr, 0, n->grads.bytes, st));
    // head
    View dy{n->dlogits.ptr, HEAD, 0};
    View dx = v(n->dDb[0], 32);
    PHX_TRY(layer_bwd(n, 18, v(n->Db[0], 32), dy, &dx, s, 0));
    // decoder, top level down to the bottleneck
    for (int l = 0; l < 4; l++) {
        const int C = LEVEL_CH[l], d = 10 + 2 * (3 - l);
        PHX_TRY(relu_bwd(n, v(n->Db[l], C), v(n->dDb[l], C), C, s, l));
        View dda = v(n->dDa[l], C);
        PHX_TRY(layer_bwd(n, d + 1, v(n->Da[l], C), v(n->dDb[l], C), &dda, s, l));
        PHX_TRY(relu_bwd(n, v(n->Da[l], C), dda, C, s, l));
        View dcat = v(n->dcat[l], CAT_CH[l]);
        PHX_TRY(layer_bwd(n, d, v(n->cat[l], CAT_CH[l]), dda, &dcat, s, l));
        // the upsampled head channels' gradient goes to the level below
        DevMem& below = l < 3 ? n->dDb[l + 1] : n->dB4;
        PHX_TRY(phx_nn_up_bwd(n->handle, n->dcat[l].ptr, CAT_CH[l], 0, UP_CH[l], s.B, s.H >> l, s.W >> l, below.ptr));
    }
    // bottleneck
    PHX_TRY(relu_bwd(n, v(n->B4, 160), v(n->dB4, 160), 160, s, 4));
    View dA4 = v(n->dA[4], 160);
    PHX_TRY(layer_bwd(n, 9, v(n->A[4], 160), v(n->dB4, 160), &dA4, s, 4));
    PHX_TRY(relu_bwd(n, v(n->A[4], 160), dA4, 160, s, 4));
    View dp = v(n->dpool[4], 128);
    PHX_TRY(layer_bwd(n, 8, v(n->pool[4], 128), dA4, &dp, s, 4));
    // encoder, bottom level up
    for (int l = 3; l >= 0; l--) {
        const int C = LEVEL_CH[l];
        // pooling's gradient joins the skip gradient the decoder wrote
        PHX_TRY(phx_nn_pool_bwd(n->handle, n->dpool[l + 1].ptr, C, s.B, s.H >> l, s.W >> l, n->dcat[l].ptr, CAT_CH[l],
                                UP_CH[l]));
        View y = v(n->cat[l], CAT_CH[l], UP_CH[l]);
        View dyb = v(n->dcat[l], CAT_CH[l], UP_CH[l]);
        PHX_TRY(relu_bwd(n, y, dyb, C, s, l));
        View dA = v(n->dA[l], C);
        PHX_TRY(layer_bwd(n, 2 * l + 1, v(n->A[l], C), dyb, &dA, s, l));
        PHX_TRY(relu_bwd(n, v(n->A[l], C), dA, C, s, l));
        if (l > 0) {
            View dpl = v(n->dpool[l], LEVEL_CH[l - 1]);
            PHX_TRY(layer_bwd(n, 2 * l, v(n->pool[l], LEVEL_CH[l - 1]), dA, &dpl, s, l));
        } else {
            PHX_TRY(layer_bwd(n, 0, View{(void*)feat, FEAT, 0}, dA, nullptr, s, 0));
        }
    }
    return PHX_OK;
}

int32_t flip_all(phx_unet_s* n) {
    for (int i = 1; i < NL; i++) {
        Conv& c = n->L[i];
        PHX_TRY(phx_nn_flip(n->handle, c.wb.ptr, c.cout, c.cin, c.Kp, c.w2.ptr, c.Kp2));
    }
    return PHX_OK;
}

// Host blob layout per layer: W [cout][9 cin] (k = tap * cin + ci), then b [cout].
uint64_t blob_count() {
    uint64_t t = 0;
    for (int i = 0; i < NL; i++) t += (uint64_t)COUT[i] * 9 * CIN[i] + COUT[i];
    return t;
}

// Uploads the fp32 master weights from a host blob, zeroes the Adam moments,
// writes the bf16 copies and the flipped data-gradient weights.
int32_t load(phx_unet_s* n, const float* blob) {
    cudaStream_t st = n->ctx->stream;
    const float* q = blob;
    for (int i = 0; i < NL; i++) {
        Conv& c = n->L[i];
        std::vector<float> w((size_t)c.cout * c.Kp, 0.0f);
        for (int r = 0; r < c.cout; r++) memcpy(&w[(size_t)r * c.Kp], q + (size_t)r * c.K, c.K * sizeof(float));
        q += (size_t)c.cout * c.K;
        PHX_CUDA(cudaMemcpyAsync(c.w32.ptr, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        PHX_CUDA(cudaMemcpyAsync(c.b32.ptr, q, c.cout * sizeof(float), cudaMemcpyHostToDevice, st));
        q += c.cout;
        // The transfers are from pageable memory and complete before return.
        PHX_CUDA(cudaStreamSynchronize(st));
        PHX_CUDA(cudaMemsetAsync(c.mw.ptr, 0, c.mw.bytes, st));
        PHX_CUDA(cudaMemsetAsync(c.vw.ptr, 0, c.vw.bytes, st));
        PHX_CUDA(cudaMemsetAsync(c.mb.ptr, 0, c.mb.bytes, st));
        PHX_CUDA(cudaMemsetAsync(c.vb.ptr, 0, c.vb.bytes, st));
        // bf16 copy: an Adam step of rate 0 with a zero gradient
        PHX_CUDA(cudaMemsetAsync(c.gw, 0, (size_t)c.cout * c.Kp * sizeof(float), st));
        PHX_TRY(phx_nn_adam(n->handle, (float*)c.w32.ptr, c.gw, (float*)c.mw.ptr, (float*)c.vw.ptr,
                            c.wb.ptr, c.cout, c.Kp, c.K, 1, 0.0f, n->b1, n->b2, n->eps, 1));
    }
    n->step = 0;
    return flip_all(n);
}

// splitmix64 + Box-Muller, so the initial weights are one function of the seed.
struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u = uniform(), w = uniform();
        return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * w);
    }
};

std::vector<float> init_blob(uint64_t seed) {
    std::vector<float> b(blob_count());
    Rng r{seed};
    size_t o = 0;
    for (int i = 0; i < NL; i++) {
        const int K = 9 * CIN[i];
        // He initialisation; the head starts near a uniform 5 x 5 box filter.
        const double sd = i == NL - 1 ? 1e-3 : std::sqrt(2.0 / K);
        for (int j = 0; j < COUT[i] * K; j++) b[o++] = (float)(sd * r.normal());
        for (int j = 0; j < COUT[i]; j++) b[o++] = (i == NL - 1 && j == 25) ? -4.6f : 0.0f;
    }
    return b;
}

int32_t check_shape(const Shape& s) {
    if (s.B <= 0 || s.H <= 0 || s.W <= 0 || s.H % 16 || s.W % 16)
        return fail(PHX_ERR_INVALID, "unet: image %dx%d (x%d) must be a positive multiple of 16", s.W, s.H, s.B);
    if ((uint64_t)s.B * s.H * s.W > (1ull << 27)) return fail(PHX_ERR_INVALID, "unet: image too large");
    return PHX_OK;
}

// Pixel (x, y) of the image mirrored by `flip` (bit 0: in x, bit 1: in y);
// padding outside w x h stays where it is.
__device__ __forceinline__ size_t mirrored(int x, int y, int w, int h, int Wp, int flip) {
    if (x < w && y < h) {
        if (flip & 1) x = w - 1 - x;
        if (flip & 2) y = h - 1 - y;
    }
    return (size_t)y * Wp + x;
}

// The network's inputs of the mirrored image: features (FEAT bf16 a pixel,
// moved as 16-bit words), irradiance and albedo (3 floats a pixel).
__global__ void k_flip_inputs(const uint4* __restrict__ feat, const float* __restrict__ irr,
                              const float* __restrict__ alb, uint4* __restrict__ ffeat, float* __restrict__ firr,
                              float* __restrict__ falb, int w, int h, int Hp, int Wp, int flip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Hp * Wp) return;
    const int x = i % Wp, y = i / Wp;
    const size_t j = mirrored(x, y, w, h, Wp, flip);
    static_assert(FEAT * 2 == 2 * sizeof(uint4), "a pixel's features are two uint4");
    ffeat[2 * (size_t)i] = feat[2 * j];
    ffeat[2 * (size_t)i + 1] = feat[2 * j + 1];
    for (int c = 0; c < 3; c++) {
        firr[3 * (size_t)i + c] = irr[3 * j + c];
        falb[3 * (size_t)i + c] = alb[3 * j + c];
    }
}

// Adds the mirrored image's filtered result and error estimate back in the
// frame's own pixel order; `scale` on the last image makes the sum a mean.
__global__ void k_flip_add(float* __restrict__ out, float* __restrict__ err, const float* __restrict__ fout,
                           const float* __restrict__ ferr, int w, int h, int Wp, int flip, float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int x = i % w, y = i / w;
    const size_t p = (size_t)y * Wp + x;
    const size_t j = mirrored(x, y, w, h, Wp, flip);
    for (int c = 0; c < 3; c++) out[3 * p + c] = (out[3 * p + c] + fout[3 * j + c]) * scale;
    err[p] = (err[p] + ferr[j]) * scale;
}

}  // namespace
}  // namespace phx

using namespace phx;

extern "C" {

int32_t phx_unet_create(phx_ctx ctx, uint64_t seed, phx_unet* out) {
    if (!ctx || !out) return fail(PHX_ERR_INVALID, "null argument");
    *out = nullptr;
    PHX_TRY(use(&ctx->c));
    phx_unet_s* n = new phx_unet_s();
    n->handle = ctx;
    n->ctx = &ctx->c;
    int32_t rc = PHX_OK;
    for (int i = 0; i < NL && rc == PHX_OK; i++) {
        Conv& c = n->L[i];
        c.cin = CIN[i];
        c.cout = COUT[i];
        c.K = 9 * c.cin;
        c.Kp = round64(c.K);
        c.Kp2 = round64(9 * c.cout);
        const size_t W = (size_t)c.cout * c.Kp;
        if ((rc = c.w32.reserve(W * 4)) < 0 || (rc = c.wb.reserve(W * 2)) < 0 || (rc = c.mw.reserve(W * 4)) < 0 ||
            (rc = c.vw.reserve(W * 4)) < 0 || (rc = c.b32.reserve(c.cout * 4)) < 0 ||
            (rc = c.mb.reserve(c.cout * 4)) < 0 || (rc = c.vb.reserve(c.cout * 4)) < 0 ||
            (rc = c.w2.reserve((size_t)c.cin * c.Kp2 * 2)) < 0)
            break;
    }
    if (rc == PHX_OK) {
        size_t off_w[NL], off_b[NL];
        const size_t total = grad_layout(off_w, off_b);
        rc = n->grads.reserve(total * sizeof(float));
        if (rc == PHX_OK) rc = cuda_check(cudaMemsetAsync(n->grads.ptr, 0, total * sizeof(float), ctx->c.stream), "grads");
        for (int i = 0; i < NL && rc == PHX_OK; i++) {
            n->L[i].gw = (float*)n->grads.ptr + off_w[i];
            n->L[i].gb = (float*)n->grads.ptr + off_b[i];
        }
    }
    if (rc == PHX_OK && (rc = n->zero_bias.reserve(288 * 4)) == PHX_OK)
        rc = cuda_check(cudaMemsetAsync(n->zero_bias.ptr, 0, 288 * 4, ctx->c.stream), "zero bias");
    if (rc == PHX_OK) rc = load(n, init_blob(seed).data());
    if (rc == PHX_OK) rc = wait_stream(ctx->c.stream, PHX_DEFAULT_WAIT_MS);
    if (rc < 0) {
        delete n;
        return rc;
    }
    ctx->c.live++;
    *out = n;
    return PHX_OK;
}

int32_t phx_unet_destroy(phx_unet net) {
    if (!net) return PHX_OK;
    Ctx* c = net->ctx;
    if (use(c) == PHX_OK) cudaStreamSynchronize(c->stream);
    delete net;
    c->live--;
    return PHX_OK;
}

int32_t phx_unet_param_count(phx_unet net, uint64_t* count) {
    if (!net || !count) return fail(PHX_ERR_INVALID, "null argument");
    *count = blob_count();
    return PHX_OK;
}

int32_t phx_unet_set_params(phx_unet net, const float* params, uint64_t count) {
    if (!net || !params) return fail(PHX_ERR_INVALID, "null argument");
    if (count != blob_count()) return fail(PHX_ERR_INVALID, "unet: %llu parameters, expected %llu",
                                           (unsigned long long)count, (unsigned long long)blob_count());
    PHX_TRY(use(net->ctx));
    PHX_TRY(load(net, params));
    return wait_stream(net->ctx->stream, PHX_DEFAULT_WAIT_MS);
}

// Reads the fp32 master weights (which = 0) or the last gradients (which = 1)
// in the blob layout. Synchronous.
int32_t phx_unet_get(phx_unet net, int32_t which, float* dst, uint64_t count) {
    if (!net || !dst || (which != 0 && which != 1)) return fail(PHX_ERR_INVALID, "unet get arguments");
    if (count != blob_count()) return fail(PHX_ERR_INVALID, "unet: %llu parameters, expected %llu",
                                           (unsigned long long)count, (unsigned long long)blob_count());
    PHX_TRY(use(net->ctx));
    PHX_TRY(wait_stream(net->ctx->stream, PHX_DEFAULT_WAIT_MS));
    float* q = dst;
    for (int i = 0; i < NL; i++) {
        Conv& c = net->L[i];
        std::vector<float> w((size_t)c.cout * c.Kp);
        PHX_CUDA(cudaMemcpy(w.data(), which == 0 ? c.w32.ptr : (const void*)c.gw, w.size() * 4, cudaMemcpyDeviceToHost));
        for (int r = 0; r < c.cout; r++)
            for (int k = 0; k < c.K; k++)
                q[(size_t)r * c.K + k] = which == 0 ? w[(size_t)r * c.Kp + k] : w[(size_t)k * c.cout + r];
        q += (size_t)c.cout * c.K;
        PHX_CUDA(cudaMemcpy(q, which == 0 ? c.b32.ptr : (const void*)c.gb, c.cout * 4, cudaMemcpyDeviceToHost));
        q += c.cout;
    }
    return PHX_OK;
}

int32_t phx_unet_forward(phx_unet net, const void* feat, const float* irr, const float* alb, int32_t B, int32_t Hp,
                         int32_t Wp, int32_t h, int32_t w, float* out, float* err) {
    if (!net || !feat || !irr || !alb) return fail(PHX_ERR_INVALID, "null argument");
    Shape s{B, Hp, Wp, net->shape.train && net->shape.B == B && net->shape.H == Hp && net->shape.W == Wp};
    PHX_TRY(check_shape(s));
    PHX_TRY(use(net->ctx));
    PHX_TRY(ensure(net, s));
    if (out && err) {
        // inference: the head's epilogue applies the predicted kernels (no logits)
        PHX_TRY(forward(net, feat, s, false));
        const Conv& c = net->L[NL - 1];
        return phx_nn_conv_kpn(net->handle, net->Db[0].ptr, 32, 0, c.cin, c.wb.ptr, c.Kp, (const float*)c.b32.ptr,
                               irr, alb, B, Hp, Wp, h, w, out, err);
    }
    PHX_TRY(forward(net, feat, s));
    if (!out && !err) return PHX_OK;
    return phx_nn_kpn(net->handle, (const float*)net->logits.ptr, irr, alb, nullptr, B, Hp, Wp, h, w, out, err,
                      nullptr, nullptr, 0.0f);
}

int32_t phx_unet_grads(phx_unet net, const void* feat, const float* irr, const float* alb, const float* ref, int32_t B,
                       int32_t Hp, int32_t Wp, int32_t h, int32_t w, float err_weight, float* loss) {
    if (!net || !feat || !irr || !alb || !ref) return fail(PHX_ERR_INVALID, "null argument");
    Shape s{B, Hp, Wp, true};
    PHX_TRY(check_shape(s));
    PHX_TRY(use(net->ctx));
    PHX_TRY(ensure(net, s));
    PHX_TRY(forward(net, feat, s));
    PHX_TRY(phx_nn_kpn(net->handle, (const float*)net->logits.ptr, irr, alb, ref, B, Hp, Wp, h, w, nullptr, nullptr,
                       net->dlogits.ptr, loss, err_weight));
    return backward(net, feat, s);
}

int32_t phx_unet_adam(phx_unet net, float lr) {
    if (!net) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(net->ctx));
    const int t = ++net->step;
    for (int i = 0; i < NL; i++) {
        Conv& c = net->L[i];
        PHX_TRY(phx_nn_adam(net->handle, (float*)c.w32.ptr, c.gw, (float*)c.mw.ptr,
                            (float*)c.vw.ptr, c.wb.ptr, c.cout, c.Kp, c.K, 1, lr, net->b1, net->b2, net->eps, t));
        PHX_TRY(phx_nn_adam(net->handle, (float*)c.b32.ptr, c.gb, (float*)c.mb.ptr,
                            (float*)c.vb.ptr, nullptr, 1, c.cout, c.cout, 0, lr, net->b1, net->b2, net->eps, t));
    }
    return flip_all(net);
}

int32_t phx_unet_train_step(phx_unet net, const void* feat, const float* irr, const float* alb, const float* ref,
                            int32_t B, int32_t Hp, int32_t Wp, int32_t h, int32_t w, float err_weight, float lr,
                            float* loss) {
    PHX_TRY(phx_unet_grads(net, feat, irr, alb, ref, B, Hp, Wp, h, w, err_weight, loss));
    return phx_unet_adam(net, lr);
}

int32_t phx_unet_grad_arena(phx_unet net, float** grads, uint64_t* count) {
    if (!net || !grads || !count) return fail(PHX_ERR_INVALID, "null argument");
    *grads = (float*)net->grads.ptr;
    *count = grad_layout(nullptr, nullptr);
    return PHX_OK;
}

int32_t phx_unet_logits(phx_unet net, float** logits) {
    if (!net || !logits) return fail(PHX_ERR_INVALID, "null argument");
    *logits = (float*)net->logits.ptr;
    return PHX_OK;
}

int32_t phx_unet_set_clamp(phx_unet net, int32_t on) {
    if (!net) return fail(PHX_ERR_INVALID, "null network");
    net->clamp = on != 0;
    return PHX_OK;
}

int32_t phx_unet_set_flips(phx_unet net, int32_t images) {
    if (!net) return fail(PHX_ERR_INVALID, "null network");
    if (images != 1 && images != 2 && images != 4) return fail(PHX_ERR_INVALID, "unet: flips %d (1, 2 or 4)", images);
    net->flips = images;
    return PHX_OK;
}

int32_t phx_unet_denoise_px(phx_unet net, uint32_t* px, const float* half, uint32_t w, uint32_t h,
                            const float view[4], int32_t tile, float threshold, int32_t keep, uint32_t* fallback) {
    if (!net || !px || !view) return fail(PHX_ERR_INVALID, "null argument");
    if (w == 0 || h == 0) return PHX_OK;
    if (tile <= 0) return fail(PHX_ERR_INVALID, "unet: tile %d", tile);
    PHX_TRY(use(net->ctx));
    const int Hp = (int)((h + 15) / 16 * 16), Wp = (int)((w + 15) / 16 * 16);
    const size_t P = (size_t)Hp * Wp;
    PHX_TRY(net->feat.reserve(P * FEAT * 2));
    PHX_TRY(net->irr.reserve(P * 12));
    PHX_TRY(net->alb.reserve(P * 12));
    PHX_TRY(net->out.reserve(P * 12));
    PHX_TRY(net->err.reserve(P * 4));
    PHX_TRY(net->tile_err.reserve((size_t)((w + tile - 1) / tile) * ((h + tile - 1) / tile) * 4));
    PHX_TRY(net->fallback.reserve(4));
    PHX_TRY(phx_nn_features(net->handle, px, half, (int)w, (int)h, Hp, Wp, net->feat.ptr, (float*)net->irr.ptr,
                            (float*)net->alb.ptr));
    // With the clamp on, the network reads the features as they are and the
    // kernels it predicts filter the irradiance after the a-trous firefly
    // clamp (off by default: on the C2 frame at 24-40 spp it raised relMSE
    // by about 1 %: the network already gives lone bright samples little
    // weight, and the clamp also darkens true highlights).
    const float* filtered = (const float*)net->irr.ptr;
    if (net->clamp) {
        PHX_TRY(net->irr_clamped.reserve(P * 12));
        PHX_TRY(phx_nn_firefly(net->handle, filtered, (float*)net->irr_clamped.ptr, 1, Hp, Wp, (int)h, (int)w));
        filtered = (const float*)net->irr_clamped.ptr;
    }
    PHX_TRY(phx_unet_forward(net, net->feat.ptr, filtered, (const float*)net->alb.ptr, 1, Hp, Wp, (int)h, (int)w,
                             (float*)net->out.ptr, (float*)net->err.ptr));
    // The mean over mirrored images (the network trained on mirrored crops):
    // each mirrored image's kernels filter its own mirrored irradiance.
    for (int f = 1; f < net->flips; f++) {
        if (f == 1) {
            PHX_TRY(net->ffeat.reserve(P * FEAT * 2));
            PHX_TRY(net->firr.reserve(P * 12));
            PHX_TRY(net->falb.reserve(P * 12));
            PHX_TRY(net->fout.reserve(P * 12));
            PHX_TRY(net->ferr.reserve(P * 4));
        }
        cudaStream_t s = net->ctx->stream;
        k_flip_inputs<<<(int)((P + 255) / 256), 256, 0, s>>>((const uint4*)net->feat.ptr, filtered,
                                                              (const float*)net->alb.ptr, (uint4*)net->ffeat.ptr,
                                                              (float*)net->firr.ptr, (float*)net->falb.ptr, (int)w,
                                                              (int)h, Hp, Wp, f);
        PHX_CUDA(cudaGetLastError());
        PHX_TRY(phx_unet_forward(net, net->ffeat.ptr, (const float*)net->firr.ptr, (const float*)net->falb.ptr, 1, Hp,
                                 Wp, (int)h, (int)w, (float*)net->fout.ptr, (float*)net->ferr.ptr));
        const float scale = f + 1 == net->flips ? 1.0f / (float)net->flips : 1.0f;
        k_flip_add<<<(int)(((size_t)w * h + 255) / 256), 256, 0, s>>>((float*)net->out.ptr, (float*)net->err.ptr,
                                                                      (const float*)net->fout.ptr,
                                                                      (const float*)net->ferr.ptr, (int)w, (int)h, Wp,
                                                                      f, scale);
        PHX_CUDA(cudaGetLastError());
    }
    // The a-trous filter everywhere first; the learned result then replaces it
    // on every tile whose estimate is within the threshold.
    const float strength[4] = {64.0f, 8.0f, 40.0f, 7.0f};
    PHX_TRY(phx_denoise(net->handle, px, w, h, strength, view, keep));
    PHX_TRY(phx_nn_compose(net->handle, px, (int)w, (int)h, Wp, (const float*)net->out.ptr,
                           (const float*)net->err.ptr, tile, threshold, keep, view[1], view[2],
                           (float*)net->tile_err.ptr, (uint32_t*)net->fallback.ptr));
    if (!fallback) return PHX_OK;
    PHX_TRY(wait_stream(net->ctx->stream, PHX_DEFAULT_WAIT_MS));
    return cuda_check(cudaMemcpy(fallback, net->fallback.ptr, 4, cudaMemcpyDeviceToHost), "fallback count");
}

}  // extern "C"
