// Edge-avoiding a-trous denoiser (phiray kernel::Denoise,
// src/kernel/denoise.wgsl:1-134, driven as Tracer::denoise_with,
// src/trace/read.rs:85-119: four rounds at steps 1, 2, 4, 8).
//
// Fast path (phx_denoise): one prep kernel turns each pixel's sums into its
// guides once — display-space albedo, unit normal, mean depth, 1/count and
// the demodulated radiance — as float4 planes in a context scratch, and the
// four rounds ping-pong float4 images there. The reference recomputes every
// tap's guides (three pows for the albedo alone) 25 times a round; these are
// the same values, computed once, so the output is unchanged bit for bit.
// The final round writes phiray's planes: linear sums (1n..4n, unless keep),
// shown colour (4n..7n) and the packed pixel (0..n). Planes 14n..20n, the
// reference's ping-pong scratch, are not touched.
//
// Pass path (PHX_KERNEL_DENOISE): the shader as written, one round per step
// over the px buffer alone, planes 14n/17n included.
#include "internal.cuh"
#include "vec.cuh"

namespace phx {
namespace {

__device__ __forceinline__ float luma_of(f3 c) { return dot(c, mk(0.2126f, 0.7152f, 0.0722f)); }
__device__ __forceinline__ float fat(const uint32_t* px, uint32_t i) { return __uint_as_float(px[i]); }
__device__ __forceinline__ f3 v3at(const uint32_t* px, uint32_t base, uint32_t i) {
    const uint32_t o = base + 3 * i;
    return mk(fat(px, o), fat(px, o + 1), fat(px, o + 2));
}
__device__ __forceinline__ void put3(uint32_t* px, uint32_t base, uint32_t i, f3 v) {
    const uint32_t o = base + 3 * i;
    px[o] = __float_as_uint(v.x);
    px[o + 1] = __float_as_uint(v.y);
    px[o + 2] = __float_as_uint(v.z);
}
__device__ __forceinline__ float inv_count(const uint32_t* px, uint32_t n, uint32_t i) {
    const uint32_t c = px[31 * n + i];
    return 1.0f / (float)(c > 1 ? c : 1);
}
__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }

__constant__ float KERNEL3[3] = {0.375f, 0.25f, 0.0625f};

// denoise.wgsl:23-39, once per pixel.
__global__ void __launch_bounds__(256) k_prep(const uint32_t* __restrict__ px, uint32_t n, float4* __restrict__ g0,
                                              float4* __restrict__ g1, float4* __restrict__ a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float k = inv_count(px, n, i);
    const f3 albedo = srgb(v3at(px, 7 * n, i) * k);
    const f3 normal = normalize(v3at(px, 10 * n, i) + mk(1e-9f));
    const float depth = fat(px, 13 * n + i) * k;
    const f3 demod = v3at(px, 1 * n, i) * k / vmax(albedo, mk(0.05f));
    g0[i] = make_float4(albedo.x, albedo.y, albedo.z, depth);
    g1[i] = make_float4(normal.x, normal.y, normal.z, k);
    a[i] = make_float4(demod.x, demod.y, demod.z, 0.0f);
}

struct RoundArgs {
    uint32_t w, h, n, step, keep;
    float s0, s1, s2, s3;
    float exposure, gamma;
};

// denoise.wgsl:47-134, one round, guides from the prep planes.
template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(256) k_round(const float4* __restrict__ g0, const float4* __restrict__ g1,
                                               const float4* __restrict__ in, float4* __restrict__ out, uint32_t* px,
                                               RoundArgs p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= (int)p.w || y >= (int)p.h) return;
    const uint32_t i = (uint32_t)y * p.w + (uint32_t)x;
    f3 centre = xyz(__ldg(in + i));
    if (FIRST) {
        float near_top = 0.0f;
        f3 near_sum = mk(0.0f);
        float near_n = 0.0f;
        for (int dy = -1; dy <= 1; dy++) {
            for (int dx = -1; dx <= 1; dx++) {
                const int sx = x + dx, sy = y + dy;
                if ((dx == 0 && dy == 0) || sx < 0 || sy < 0 || sx >= (int)p.w || sy >= (int)p.h) continue;
                const f3 c = xyz(__ldg(in + (uint32_t)sy * p.w + (uint32_t)sx));
                near_top = fmaxf(near_top, luma_of(c));
                near_sum += c;
                near_n += 1.0f;
            }
        }
        if (near_n > 0.0f && luma_of(centre) > 1.5f * near_top + 0.05f) centre = near_sum / near_n;
    }
    const float4 c0 = __ldg(g0 + i), c1 = __ldg(g1 + i);
    const f3 cn = xyz(c1), ca = xyz(c0);
    const float cd = c0.w;
    const float lc = luma_of(centre);
    f3 sum = mk(0.0f);
    float weight = 0.0f;
    for (int dy = -2; dy <= 2; dy++) {
        const int sy = y + dy * (int)p.step;
        if (sy < 0 || sy >= (int)p.h) continue;
        for (int dx = -2; dx <= 2; dx++) {
            const int sx = x + dx * (int)p.step;
            if (sx < 0 || sx >= (int)p.w) continue;
            const uint32_t j = (uint32_t)sy * p.w + (uint32_t)sx;
            const float4 j0 = __ldg(g0 + j);
            if ((j0.w < 0.0f) != (cd < 0.0f)) continue;
            const f3 tap = (j == i) ? centre : xyz(__ldg(in + j));
            const float4 j1 = __ldg(g1 + j);
            const float dn = fmaxf(0.0f, 1.0f - dot(cn, xyz(j1)));
            const float da = length(xyz(j0) - ca);
            const float dd = fabsf(j0.w - cd) / fmaxf(fabsf(cd), 1e-3f);
            const float dl = fabsf(luma_of(tap) - lc) / (0.08f + lc);
            const float stop = pm_exp(-dn * p.s0 - da * p.s1 - dd * p.s2 - dl * dl * p.s3);
            const float k = KERNEL3[dx < 0 ? -dx : dx] * KERNEL3[dy < 0 ? -dy : dy];
            sum += tap * k * stop;
            weight += k * stop;
        }
    }
    const f3 o = weight > 0.0f ? sum / weight : centre;
    if (!LAST) {
        out[i] = make_float4(o.x, o.y, o.z, 0.0f);
        return;
    }
    const uint32_t n = p.n;
    const float k = c1.w;
    const float met = 1.0f - fat(px, 33 * n + i) * k;
    const f3 lin = (met > 0.5f * k) ? o * vmax(ca, mk(0.05f)) : mk(0.0f);
    if (p.keep == 0) put3(px, 1 * n, i, lin / k);
    const float cov = fat(px, 23 * n + i) * k;
    const f3 grid = v3at(px, 20 * n, i) * k;
    const f3 shown = view_transform_std(lin / fmaxf(met, k), p.exposure, p.gamma) * (1.0f - cov) + grid;
    put3(px, 4 * n, i, shown);
    px[i] = pack_rgba(shown, fat(px, 24 * n + i) * k);
}

// ---- the shader as written, for Pass replay (one round per step) ----

struct PxView {
    uint32_t* px;
    uint32_t n, round;
    __device__ float inv_n(uint32_t i) const { return inv_count(px, n, i); }
    __device__ f3 albedo_of(uint32_t i) const { return srgb(v3at(px, 7 * n, i) * inv_n(i)); }
    __device__ f3 normal_of(uint32_t i) const { return normalize(v3at(px, 10 * n, i) + mk(1e-9f)); }
    __device__ float depth_of(uint32_t i) const { return fat(px, 13 * n + i) * inv_n(i); }
    __device__ f3 demodulated(uint32_t i) const { return v3at(px, 1 * n, i) * inv_n(i) / vmax(albedo_of(i), mk(0.05f)); }
    __device__ f3 read_in(uint32_t i) const {
        if (round == 0) return demodulated(i);
        return v3at(px, ((round & 1) == 1 ? 14u : 17u) * n, i);
    }
};

__global__ void __launch_bounds__(256) k_denoise_px(phx_denoise_param p, uint32_t* px, uint32_t items) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n || i >= items) return;
    PxView v{px, p.n, p.round};
    const int x = (int)(i % p.w), y = (int)(i / p.w);
    f3 centre = v.read_in(i);
    if (p.round == 0) {
        float near_top = 0.0f;
        f3 near_sum = mk(0.0f);
        float near_n = 0.0f;
        for (int dy = -1; dy <= 1; dy++) {
            for (int dx = -1; dx <= 1; dx++) {
                const int sx = x + dx, sy = y + dy;
                if ((dx == 0 && dy == 0) || sx < 0 || sy < 0 || sx >= (int)p.w || sy >= (int)p.h) continue;
                const f3 c = v.read_in((uint32_t)sy * p.w + (uint32_t)sx);
                near_top = fmaxf(near_top, luma_of(c));
                near_sum += c;
                near_n += 1.0f;
            }
        }
        if (near_n > 0.0f && luma_of(centre) > 1.5f * near_top + 0.05f) centre = near_sum / near_n;
    }
    const f3 cn = v.normal_of(i);
    const f3 ca = v.albedo_of(i);
    const float cd = v.depth_of(i);
    const float lc = luma_of(centre);
    f3 sum = mk(0.0f);
    float weight = 0.0f;
    for (int dy = -2; dy <= 2; dy++) {
        for (int dx = -2; dx <= 2; dx++) {
            const int sx = x + dx * (int)p.step, sy = y + dy * (int)p.step;
            if (sx < 0 || sy < 0 || sx >= (int)p.w || sy >= (int)p.h) continue;
            const uint32_t j = (uint32_t)sy * p.w + (uint32_t)sx;
            if ((v.depth_of(j) < 0.0f) != (cd < 0.0f)) continue;
            const f3 tap = (j == i) ? centre : v.read_in(j);
            const float dn = fmaxf(0.0f, 1.0f - dot(cn, v.normal_of(j)));
            const float da = length(v.albedo_of(j) - ca);
            const float dd = fabsf(v.depth_of(j) - cd) / fmaxf(fabsf(cd), 1e-3f);
            const float dl = fabsf(luma_of(tap) - lc) / (0.08f + lc);
            const float stop = pm_exp(-dn * p.strength[0] - da * p.strength[1] - dd * p.strength[2] -
                                      dl * dl * p.strength[3]);
            const float k = KERNEL3[dx < 0 ? -dx : dx] * KERNEL3[dy < 0 ? -dy : dy];
            sum += tap * k * stop;
            weight += k * stop;
        }
    }
    const f3 o = weight > 0.0f ? sum / weight : centre;
    if (p.last == 0) {
        put3(px, ((p.round & 1) == 1 ? 17u : 14u) * p.n, i, o);
        return;
    }
    const uint32_t n = p.n;
    const float k = v.inv_n(i);
    const float met = 1.0f - fat(px, 33 * n + i) * k;
    const f3 lin = (met > 0.5f * k) ? o * vmax(v.albedo_of(i), mk(0.05f)) : mk(0.0f);
    if (p.keep == 0) put3(px, 1 * n, i, lin / k);
    const float cov = fat(px, 23 * n + i) * k;
    const f3 grid = v3at(px, 20 * n, i) * k;
    const f3 shown = view_transform_std(lin / fmaxf(met, k), p.view[1], p.view[2]) * (1.0f - cov) + grid;
    put3(px, 4 * n, i, shown);
    px[i] = pack_rgba(shown, fat(px, 24 * n + i) * k);
}

}  // namespace

int32_t launch_denoise_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items) {
    phx_denoise_param p;
    memcpy(&p, params, sizeof p);
    if (p.view[0] != 0.0f) return fail(PHX_ERR_INVALID, "denoise: only the Standard view transform is supported");
    if (p.n == 0 || items == 0) return PHX_OK;
    if (p.n != p.w * p.h) return fail(PHX_ERR_INVALID, "denoise: n %u != w*h", p.n);
    k_denoise_px<<<(items + 255) / 256, 256, 0, s>>>(p, (uint32_t*)bufs[0], items);
    return cuda_check(cudaGetLastError(), "denoise step");
}

int32_t enqueue_denoise(Ctx* c, DevMem& scratch, uint32_t* px, uint32_t w, uint32_t h, const float strength[4],
                        const float view[4], int32_t keep) {
    if (view[0] != 0.0f) return fail(PHX_ERR_INVALID, "denoise: only the Standard view transform is supported");
    const uint64_t n = (uint64_t)w * h;
    if (n == 0) return PHX_OK;
    if (n > 0x7FFFFFFFull / 34) return fail(PHX_ERR_INVALID, "denoise: %ux%u is too large", w, h);
    PHX_TRY(scratch.reserve(n * 16 * 4));
    float4* g0 = (float4*)scratch.ptr;
    float4* g1 = g0 + n;
    float4* a = g1 + n;
    float4* b = a + n;
    cudaStream_t s = c->stream;
    k_prep<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(px, (uint32_t)n, g0, g1, a);
    RoundArgs p{w, h, (uint32_t)n, 1, keep ? 1u : 0u, strength[0], strength[1], strength[2], strength[3], view[1], view[2]};
    const dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    p.step = 1;
    k_round<true, false><<<grid, block, 0, s>>>(g0, g1, a, b, px, p);
    p.step = 2;
    k_round<false, false><<<grid, block, 0, s>>>(g0, g1, b, a, px, p);
    p.step = 4;
    k_round<false, false><<<grid, block, 0, s>>>(g0, g1, a, b, px, p);
    p.step = 8;
    k_round<false, true><<<grid, block, 0, s>>>(g0, g1, b, nullptr, px, p);
    return cuda_check(cudaGetLastError(), "denoise");
}

}  // namespace phx

using namespace phx;

extern "C" int32_t phx_denoise(phx_ctx ctx, uint32_t* px, uint32_t w, uint32_t h, const float strength[4],
                               const float view[4], int32_t keep) {
    if (!ctx || !strength || !view || (w * h && !px)) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(&ctx->c));
    return enqueue_denoise(&ctx->c, ctx->c.denoise_scratch, px, w, h, strength, view, keep);
}
