// BF16 tensor-core kernels for the learned denoiser (tcgen05, tc.cuh).
//
// phx_gemm_bf16: D (fp32, M x N) = A (bf16, M x K, row-major) x B^T (B bf16,
// N x K, row-major). The building block the convolutions stage through; also
// the engine's own parity check against a plain matrix product.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>

#include "../../include/phiray_math.h"
#include "internal.cuh"
#include "tc.cuh"
#include "vec.cuh"

namespace phx {
namespace {

using bf16 = __nv_bfloat16;

// Shared-memory plan of one CTA: the A tile, then the B tile (the rooms
// between them are spare space, zero since the descriptors were validated
// against plain matrix products).
template <int N>
struct Plan {
    static constexpr int A_BYTES = tc::BM * tc::BK * 2;
    static constexpr int B_BYTES = N * tc::BK * 2;
    static constexpr int A_ROOM = 0;
    static constexpr int B_ROOM = 0;
    static constexpr int A_OFF = 0;
    static constexpr int B_OFF = A_BYTES + A_ROOM;
    static constexpr int TOTAL = B_OFF + B_BYTES + B_ROOM;
};

// Raises a kernel's dynamic shared-memory limit (and carveout) once per device.
template <typename F>
int32_t smem_limit(F* kernel, int bytes, int device, std::atomic<uint64_t>& done) {
    const uint64_t bit = 1ull << (device & 63);
    if (done.load(std::memory_order_acquire) & bit) return PHX_OK;
    PHX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    // the largest shared-memory carveout, so that several blocks fit an SM
    PHX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    done.fetch_or(bit, std::memory_order_release);
    return PHX_OK;
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

template <int N>
__global__ void __launch_bounds__(128) k_gemm_bf16(const bf16* __restrict__ A, const bf16* __restrict__ B,
                                                   float* __restrict__ D, int M, int K, uint32_t* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    using P = Plan<N>;
    uint8_t* a_tile = smem + P::A_OFF;
    uint8_t* b_tile = smem + P::B_OFF;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(&tmem_base, tc::tmem_cols(N));
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_base;
    const int row0 = blockIdx.x * tc::BM;
    uint32_t phase = 0;
    bool ok = true;
    for (int kb = 0; kb < K && ok; kb += tc::BK) {
        for (int v = tid; v < tc::BM * 8; v += 128) {
            const int r = v >> 3, c = v & 7;
            const uint4 x = __ldg((const uint4*)(A + (size_t)(row0 + r) * K + kb + c * 8));
            *(uint4*)(a_tile + tc::tile_off(r, c * 8, tc::BM)) = x;
        }
        for (int v = tid; v < N * 8; v += 128) {
            const int r = v >> 3, c = v & 7;
            const uint4 x = __ldg((const uint4*)(B + (size_t)r * K + kb + c * 8));
            *(uint4*)(b_tile + tc::tile_off(r, c * 8, N)) = x;
        }
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            tc::mma_chunk<N>(tm, a_tile, b_tile, kb == 0);
            tc::mma_commit(&bar);
        }
        ok = tc::mbar_wait(&bar, phase);
        phase ^= 1u;
        ok = __syncthreads_and(ok);
    }
    tc::fence_after_sync();
    if (ok) {
        const int row = row0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (row < M) {
                float4* out = (float4*)(D + (size_t)row * N + c0);
                out[0] = make_float4(v[0], v[1], v[2], v[3]);
                out[1] = make_float4(v[4], v[5], v[6], v[7]);
                out[2] = make_float4(v[8], v[9], v[10], v[11]);
                out[3] = make_float4(v[12], v[13], v[14], v[15]);
            }
        }
    } else if (tid == 0) {
        atomicOr(status, STATUS_SPIN_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, tc::tmem_cols(N));
}

template <int N>
int32_t launch_gemm(Ctx* c, const bf16* A, const bf16* B, float* D, int M, int K) {
    const int smem = Plan<N>::TOTAL;
    static std::atomic<uint64_t> done{0};
    PHX_TRY(smem_limit(k_gemm_bf16<N>, smem, c->device, done));
    k_gemm_bf16<N><<<M / tc::BM, 128, smem, c->stream>>>(A, B, D, M, K, c->status);
    return cuda_check(cudaGetLastError(), "gemm bf16");
}

// ---- 3x3 convolution as implicit GEMM on the engine ----
//
// Activations are NHWC bf16 with a pixel pitch and a channel offset, so a
// layer can read one channel range of a wider buffer and write into another
// (the U-Net's skip concatenations cost no copy). Weights are [cout][Kp] bf16,
// k = (3 * ty + tx) * cin + ci, zero past K = 9 cin up to Kp (a multiple of 64).
// cin, pitches and offsets are multiples of 8 (16-byte vectors).

struct Geo {
    int B, H, W;       // images and their size (stride 1, pad 1: same size out)
    int cin, xs, xo;   // input channels, pixel pitch, channel offset
    int cout, ys, yo;  // output channels (= the tile's N), pitch, offset
    int K, Kp;         // 9 cin, padded to a multiple of 64
};

// A row of the im2col matrix: the pixel's image, y, x (or -1: past the end).
struct PixRow {
    int b, y, x;
};

__device__ __forceinline__ PixRow pix_row(int p, const Geo& g) {
    const int P = g.B * g.H * g.W;
    if (p >= P) return PixRow{-1, 0, 0};
    const int hw = g.H * g.W;
    const int b = p / hw, rem = p - b * hw;
    return PixRow{b, rem / g.W, rem - (rem / g.W) * g.W};
}

// 8 consecutive k (one tap, 8 channels) of im2col row `pr`, 16 bytes.
__device__ __forceinline__ uint4 im2col_vec(const bf16* __restrict__ X, const PixRow& pr, int k, const Geo& g) {
    if (pr.b < 0 || k >= g.K) return make_uint4(0, 0, 0, 0);
    const int tap = k / g.cin, ci = k - tap * g.cin;
    const int y = pr.y + tap / 3 - 1, x = pr.x + tap % 3 - 1;
    if (y < 0 || y >= g.H || x < 0 || x >= g.W) return make_uint4(0, 0, 0, 0);
    return __ldg((const uint4*)(X + ((size_t)(pr.b * g.H + y) * g.W + x) * g.xs + g.xo + ci));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *(const uint32_t*)&v;
}

// Asynchronous 16-byte global -> shared copy; src_bytes 0 fills zeros (the
// source address must still be a valid one, it is not read).
__device__ __forceinline__ void cp_async_ca16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_cg16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// ---- the convolution forward: shifted descriptors over a staged patch ----
//
// One CTA computes a 16 x 8 block of output pixels of one image (M = 128:
// m = 8 ty + tx, so each 8-row group of the MMA is one image row of 8
// pixels) for N output channels. Input channels are taken CC at a time: the
// (16 + 2) x (8 + 2) input patch of those channels is staged once in shared
// memory in the canonical K-major layout — 16-byte pixel vectors of 8
// channels, a patch row of 10 pixels every ROWB = 160 bytes, the 8-channel
// groups LBO = 18 * 160 bytes apart — and the A operand of tap (dy, dx) is
// the same patch seen through a descriptor whose start moves by
// dy * ROWB + dx * 16 bytes (SBO = ROWB). The nine taps' MMAs read one
// staged patch instead of nine gathered copies of it. The weights of the
// nine taps for the CC channels (B tiles N x CC each) are staged beside it.
// Chunks go through a STAGES-deep ring filled by cp.async (zero-filled
// outside the image), each stage refilled after the mbarrier of the MMAs
// that last read it.
constexpr int TY = 16, TX = 8;
constexpr int PY = TY + 2, PX = TX + 2;
constexpr int ROWB = PX * 16;  // bytes of one patch row of one 8-channel group (one 16 x 8 tile)

// T tiles side by side: the block covers 16 x 8T pixels, stages one
// (16 + 2) x (8T + 2) patch a chunk, and keeps T accumulators of N columns;
// tile t's A operand of tap (dy, dx) starts dy * ROWT + (8 t + dx) * 16 bytes
// into the patch. The weight chunk is read once for the T tiles.
template <int N, int CC, int T>
struct Conv {
    static constexpr int KG = CC / 8;                 // 8-channel groups a chunk
    static constexpr int PXT = TX * T + 2;            // patch width
    static constexpr int ROWT = PXT * 16;             // bytes of a patch row of one channel group
    static constexpr int LBO_A = PY * ROWT;           // between channel groups of the patch
    static constexpr int PATCH = KG * LBO_A;          // patch bytes
    static constexpr int BTAP = N * CC * 2;           // one tap's weight tile
    static constexpr int STAGE = (PATCH + 9 * BTAP + 127) / 128 * 128;
    static constexpr int STAGES = STAGE <= 40 * 1024 ? 3 : 2;
    static constexpr int TOTAL = STAGES * STAGE;
    static constexpr uint32_t ACC = tc::tmem_cols(N);  // accumulator stride in TMEM columns
    static constexpr uint32_t COLS = tc::tmem_cols(T * ACC);
};

// Y = act(conv3x3(X, W) + bias). OUT_F32: fp32 output (the network's head).
template <int N, int CC, int T, bool RELU, bool OUT_F32>
__global__ void __launch_bounds__(128) k_conv_fwd(const bf16* __restrict__ X, const bf16* __restrict__ Wt,
                                                  const float* __restrict__ bias, void* __restrict__ Y, Geo g,
                                                  uint32_t* status) {
    using C = Conv<N, CC, T>;
    constexpr int STAGES = C::STAGES;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar[STAGES];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(&tmem_base, C::COLS);
    if (tid == 0) {
        for (int i = 0; i < STAGES; i++) tc::mbar_init(&bar[i], 1);
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_base;
    const int tiles_x = (g.W + TX * T - 1) / (TX * T), tiles_y = (g.H + TY - 1) / TY;
    const int bx = blockIdx.x % tiles_x, by = (blockIdx.x / tiles_x) % tiles_y, img = blockIdx.x / (tiles_x * tiles_y);
    const int y0 = by * TY, x0 = bx * TX * T;
    const int nk = g.cin / CC;

    auto issue = [&](int chunk) {
        uint8_t* patch = smem + (chunk % STAGES) * C::STAGE;
        uint8_t* wb = patch + C::PATCH;
        const int c0 = chunk * CC;
        for (int v = tid; v < PY * C::PXT * C::KG; v += 128) {
            const int kg = v % C::KG, q = v / C::KG;
            const int py = q / C::PXT, px = q - py * C::PXT;
            const int y = y0 + py - 1, x = x0 + px - 1;
            const bool ok = y >= 0 && y < g.H && x >= 0 && x < g.W;
            const bf16* src = ok ? X + ((size_t)(img * g.H + y) * g.W + x) * g.xs + g.xo + c0 + kg * 8 : X;
            cp_async_ca16(patch + kg * C::LBO_A + py * C::ROWT + px * 16, src, ok ? 16u : 0u);
        }
        for (int v = tid; v < 9 * N * C::KG; v += 128) {
            const int kg = v % C::KG, q = v / C::KG;
            const int r = q % N, tap = q / N;
            cp_async_cg16(wb + tap * C::BTAP + tc::tile_off(r, kg * 8, N),
                          Wt + (size_t)r * g.Kp + tap * g.cin + c0 + kg * 8);
        }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nk) issue(s);
        cp_async_commit();
    }
    bool ok = true;
    constexpr uint32_t idesc = tc::instr_desc_bf16(tc::BM, N);
    constexpr uint32_t b_lbo = (N / 8) * 128;
    for (int chunk = 0; chunk < nk; chunk++) {
        cp_async_wait<STAGES - 2>();
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            const uint32_t patch = tc::smem_addr(smem + (chunk % STAGES) * C::STAGE);
            tc::fence_after_sync();
            const uint64_t da0 = tc::smem_desc(patch, C::LBO_A, C::ROWT);
            const uint64_t db0 = tc::smem_desc(patch + C::PATCH, b_lbo, 128);
#pragma unroll
            for (int t = 0; t < T; t++) {
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
#pragma unroll
                    for (int s = 0; s < CC / 16; s++) {
                        const uint64_t da =
                            da0 + (uint64_t)(((tap / 3) * C::ROWT + (TX * t + tap % 3) * 16 + 2 * s * C::LBO_A) >> 4);
                        const uint64_t db = db0 + (uint64_t)((tap * C::BTAP + 2 * s * b_lbo) >> 4);
                        tc::mma_bf16(tm + (uint32_t)t * C::ACC, da, db, idesc,
                                     (chunk == 0 && tap == 0 && s == 0) ? 0u : 1u);
                    }
                }
            }
            tc::mma_commit(&bar[chunk % STAGES]);
        }
        const int next = chunk + STAGES - 1;
        if (next < nk) {
            if (chunk >= 1) ok = tc::mbar_wait(&bar[(chunk - 1) % STAGES], ((chunk - 1) / STAGES) & 1) && ok;
            issue(next);
        }
        cp_async_commit();
    }
    ok = tc::mbar_wait(&bar[(nk - 1) % STAGES], ((nk - 1) / STAGES) & 1) && ok;
    ok = __syncthreads_and(ok);
    tc::fence_after_sync();
    if (ok) {
        const int m = warp * 32 + lane;
#pragma unroll 1
        for (int t = 0; t < T; t++) {
            const int y = y0 + m / TX, x = x0 + TX * t + m % TX;
            const bool live = y < g.H && x < g.W;
            const size_t p = ((size_t)img * g.H + y) * g.W + x;
#pragma unroll 1
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)t * C::ACC + (uint32_t)c0, v);
                if (!live) continue;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    v[j] += __ldg(bias + c0 + j);
                    if (RELU) v[j] = fmaxf(v[j], 0.0f);
                }
                if (OUT_F32) {
                    float4* o = (float4*)((float*)Y + p * g.ys + g.yo + c0);
#pragma unroll
                    for (int q = 0; q < 4; q++) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                } else {
                    uint4* o = (uint4*)((bf16*)Y + p * g.ys + g.yo + c0);
                    o[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                      pack_bf16x2(v[6], v[7]));
                    o[1] = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
                                      pack_bf16x2(v[14], v[15]));
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(status, STATUS_SPIN_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, C::COLS);
}

// ---- the same convolution, persistent and weight-stationary ----
//
// Used when the layer's weights (9 taps x N x cin bf16) and two input
// patches fit in shared memory. Each CTA loads the weights once and walks
// the output tiles blockIdx.x, + gridDim.x, ...; the tensor memory holds two
// accumulators of N columns (at column 0 and at the power of two >= N). Iteration i: thread 0 issues tile i's MMAs
// (9 taps x cin / 16, shifted descriptors over patch buffer i & 1) into
// accumulator i & 1 and commits them to mbarrier i & 1; meanwhile every
// thread waits for tile i - 1's MMAs, refills patch buffer (i + 1) & 1
// with tile i + 1's patch and writes tile i - 1's outputs from accumulator
// (i - 1) & 1. So the copies and the epilogue of neighbouring tiles run
// under the current tile's MMAs.
template <int N>
struct ConvWS {
    static constexpr int W_BYTES_PER_CIN = 9 * N * 2;  // x cin
    static constexpr int PATCH_PER_CIN = PY * ROWB / 8; // x cin (= 360 bytes a channel)
    static constexpr int PATCHES = 3;  // the tile being multiplied and the next two in flight
    static size_t bytes(int cin) { return (size_t)cin * (W_BYTES_PER_CIN + PATCHES * PATCH_PER_CIN); }
};

// The kernel-prediction step as a head convolution's epilogue (inference):
// the 32 head outputs of a pixel go from TMEM through the softmax and the
// 5 x 5 filter straight to out / err, and no logits are written.
struct KpnOut {
    const float* irr;
    const float* alb;
    float* out;
    float* err;
    int h, w;  // the valid corner of the padded H x W images
};

__device__ __forceinline__ void kpn_pixel(const float* lg, const KpnOut& k, int img, int y, int x, int Hp, int Wp,
                                          size_t p) {
    if (!(y < k.h && x < k.w)) {
        for (int c = 0; c < 3; c++) k.out[p * 3 + c] = 0.0f;
        k.err[p] = 0.0f;
        return;
    }
    float wt[25], mx = -3.0e38f;
#pragma unroll
    for (int t = 0; t < 25; t++) {
        wt[t] = lg[t];
        mx = fmaxf(mx, wt[t]);
    }
    float z = 0.0f;
#pragma unroll
    for (int t = 0; t < 25; t++) {
        wt[t] = pm_exp(wt[t] - mx);
        z += wt[t];
    }
    const float iz = 1.0f / z;
    float sm[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int t = 0; t < 25; t++) {
        const int yy = min(max(y + t / 5 - 2, 0), k.h - 1), xx = min(max(x + t % 5 - 2, 0), k.w - 1);
        const float* q = k.irr + ((size_t)(img * Hp + yy) * Wp + xx) * 3;
        const float wv = wt[t] * iz;
#pragma unroll
        for (int c = 0; c < 3; c++) sm[c] += wv * __ldg(q + c);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) k.out[p * 3 + c] = __ldg(k.alb + p * 3 + c) * sm[c];
    k.err[p] = fmaxf(pm_exp(lg[25]) - 1.0e-3f, 0.0f);
}

template <int N, bool RELU, bool OUT_F32, bool KPN = false>
__global__ void __launch_bounds__(128) k_conv_ws(const bf16* __restrict__ X, const bf16* __restrict__ Wt,
                                                 const float* __restrict__ bias, void* __restrict__ Y, Geo g,
                                                 uint32_t* status, KpnOut kp = KpnOut{}) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // accumulator b at column b * ACC (a power of two: aligned like a whole allocation)
    constexpr uint32_t ACC = tc::tmem_cols(N);
    constexpr uint32_t COLS = 2 * ACC;
    if (warp == 0) tc::tmem_alloc(&tmem_base, COLS);
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_base;
    const int KG = g.cin / 8;
    const int LBO_A = PY * ROWB;
    const int PATCH = KG * LBO_A;
    const int BTAP = N * g.cin * 2;
    uint8_t* wsm = smem;
    uint8_t* patch0 = smem + 9 * BTAP;
    const int tiles_x = (g.W + TX - 1) / TX, tiles_y = (g.H + TY - 1) / TY;
    const int ntiles = g.B * tiles_x * tiles_y;

    // the weights, once
    for (int v = tid; v < 9 * N * KG; v += 128) {
        const int kg = v % KG, q = v / KG;
        const int r = q % N, tap = q / N;
        cp_async_cg16(wsm + tap * BTAP + tc::tile_off(r, kg * 8, N), Wt + (size_t)r * g.Kp + tap * g.cin + kg * 8);
    }
    cp_async_commit();
    auto issue_patch = [&](int tile, int buf) {
        const int bx = tile % tiles_x, by = (tile / tiles_x) % tiles_y, img = tile / (tiles_x * tiles_y);
        const int y0 = by * TY, x0 = bx * TX;
        uint8_t* patch = patch0 + buf * PATCH;
        for (int v = tid; v < PY * PX * KG; v += 128) {
            const int kg = v % KG, q = v / KG;
            const int py = q / PX, px = q - py * PX;
            const int y = y0 + py - 1, x = x0 + px - 1;
            const bool ok = y >= 0 && y < g.H && x >= 0 && x < g.W;
            const bf16* src = ok ? X + ((size_t)(img * g.H + y) * g.W + x) * g.xs + g.xo + kg * 8 : X;
            cp_async_ca16(patch + kg * LBO_A + py * ROWB + px * 16, src, ok ? 16u : 0u);
        }
        cp_async_commit();
    };
    auto epilogue = [&](int tile, int buf) {
        const int bx = tile % tiles_x, by = (tile / tiles_x) % tiles_y, img = tile / (tiles_x * tiles_y);
        const int m = warp * 32 + lane;
        const int y = by * TY + m / TX, x = bx * TX + m % TX;
        const bool live = y < g.H && x < g.W;
        const size_t p = ((size_t)img * g.H + y) * g.W + x;
        if (KPN) {
            float lg[32];
            tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)buf * ACC, lg);
            tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)buf * ACC + 16u, lg + 16);
            if (live) {
#pragma unroll
                for (int j = 0; j < 26; j++) lg[j] += __ldg(bias + j);
                kpn_pixel(lg, kp, img, y, x, g.H, g.W, p);
            }
            tc::fence_before_sync();
            return;
        }
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)buf * ACC + (uint32_t)c0, v);
            if (!live) continue;
#pragma unroll
            for (int j = 0; j < 16; j++) {
                v[j] += __ldg(bias + c0 + j);
                if (RELU) v[j] = fmaxf(v[j], 0.0f);
            }
            if (OUT_F32) {
                float4* o = (float4*)((float*)Y + p * g.ys + g.yo + c0);
#pragma unroll
                for (int q = 0; q < 4; q++) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
                uint4* o = (uint4*)((bf16*)Y + p * g.ys + g.yo + c0);
                o[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                  pack_bf16x2(v[6], v[7]));
                o[1] = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
                                  pack_bf16x2(v[14], v[15]));
            }
        }
        tc::fence_before_sync();
    };

    constexpr uint32_t idesc = tc::instr_desc_bf16(tc::BM, N);
    constexpr uint32_t b_lbo = (N / 8) * 128;
    constexpr int NP = ConvWS<N>::PATCHES;
    bool ok = true;
    int i = 0, prev = -1;
    // Prologue: tiles 0 and 1 of this block in flight (commit groups 1, 2 after
    // the weights' group 0; an empty group stands in for a missing tile).
    for (int k = 0; k < NP - 1; k++) {
        const int t = blockIdx.x + k * gridDim.x;
        if (t < ntiles) issue_patch(t, k);
        else cp_async_commit();
    }
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, i++) {
        const int b = i & 1;
        cp_async_wait<NP - 2>();  // this thread's copies of tile i (and the weights) landed
        tc::fence_async_smem();
        __syncthreads();          // everyone's; and the last epilogue's TMEM reads
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t acc = tm + (uint32_t)b * ACC;
            // Descriptors are built once; a step along K or to another tap
            // adds its byte offset / 16 to the start-address field.
            const uint64_t da0 = tc::smem_desc(tc::smem_addr(patch0 + (i % NP) * PATCH), LBO_A, ROWB);
            const uint64_t db0 = tc::smem_desc(tc::smem_addr(wsm), b_lbo, 128);
            const uint64_t a_step = (uint64_t)((2 * LBO_A) >> 4), b_step = (uint64_t)((2 * b_lbo) >> 4);
            const int ks = g.cin / 16;
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                uint64_t da = da0 + (uint64_t)(((tap / 3) * ROWB + (tap % 3) * 16) >> 4);
                uint64_t db = db0 + (uint64_t)((tap * BTAP) >> 4);
                for (int s = 0; s < ks; s++) {
                    tc::mma_bf16(acc, da, db, idesc, (tap == 0 && s == 0) ? 0u : 1u);
                    da += a_step;
                    db += b_step;
                }
            }
            tc::mma_commit(&bar[b]);
        }
        if (i >= 1) ok = tc::mbar_wait(&bar[b ^ 1], ((i - 1) >> 1) & 1) && ok;  // tile i - 1's MMAs done
        // tile i + 2 into the patch buffer tile i - 1 used
        const int ahead = tile + (NP - 1) * gridDim.x;
        if (ahead < ntiles) issue_patch(ahead, (i + NP - 1) % NP);
        else cp_async_commit();
        if (i >= 1) {
            tc::fence_after_sync();
            epilogue(prev, b ^ 1);
        }
        prev = tile;
    }
    if (i >= 1) {
        ok = tc::mbar_wait(&bar[(i - 1) & 1], ((i - 1) >> 1) & 1) && ok;
        tc::fence_after_sync();
        epilogue(prev, (i - 1) & 1);
    }
    ok = __syncthreads_and(ok);
    if (!ok && tid == 0) atomicOr(status, STATUS_SPIN_LIMIT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, COLS);
}

// Weight gradient: dWt[k][co] += sum over pixels p of im2col(X)[p][k] dY[p][co].
// GEMM rows = k (a 128-row block per CTA), N = cout, the reduction over the
// pixel range of this CTA's split, 64 pixels a chunk; the tiles are written
// transposed from the NHWC vectors. The split partial sums meet in dWt by
// fp32 atomics. dY has pitch `dys` (cout channels at offset 0).
template <int N>
__global__ void __launch_bounds__(128) k_conv_wgrad(const bf16* __restrict__ X, const bf16* __restrict__ dY, int dys,
                                                    int dyo, float* __restrict__ dWt, Geo g, int chunk_px,
                                                    uint32_t* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    using P = Plan<N>;
    uint8_t* a_tile = smem + P::A_OFF;
    uint8_t* b_tile = smem + P::B_OFF;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(&tmem_base, tc::tmem_cols(N));
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_base;
    const int k0 = blockIdx.x * tc::BM;
    const int P0 = blockIdx.y * chunk_px;
    const int Ptot = g.B * g.H * g.W;
    const int P1 = min(P0 + chunk_px, Ptot);
    // A: this thread stages k-vector rv = tid % 16 (rows rv*8..rv*8+7) at
    // pixel columns tid / 16 + 8 j.
    const int rv = tid & 15;
    const int kv = k0 + rv * 8;
    uint32_t phase = 0;
    bool ok = true;
    for (int pb = P0; pb < P1 && ok; pb += tc::BK) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int col = (tid >> 4) + 8 * j;
            const PixRow pr = pix_row(pb + col < P1 ? pb + col : Ptot, g);
            const uint4 val = im2col_vec(X, pr, kv, g);
            const bf16* e = (const bf16*)&val;
#pragma unroll
            for (int q = 0; q < 8; q++) *(bf16*)(a_tile + tc::tile_off(rv * 8 + q, col, tc::BM)) = e[q];
        }
        for (int v = tid; v < N * 8; v += 128) {
            const int bv = v % (N / 8), col = v / (N / 8);
            const int p = pb + col;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (p < P1) val = __ldg((const uint4*)(dY + (size_t)p * dys + dyo + bv * 8));
            const bf16* e = (const bf16*)&val;
#pragma unroll
            for (int q = 0; q < 8; q++) *(bf16*)(b_tile + tc::tile_off(bv * 8 + q, col, N)) = e[q];
        }
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            tc::mma_chunk<N>(tm, a_tile, b_tile, pb == P0);
            tc::mma_commit(&bar);
        }
        ok = tc::mbar_wait(&bar, phase);
        phase ^= 1u;
        ok = __syncthreads_and(ok);
    }
    tc::fence_after_sync();
    if (ok && P0 < P1) {
        const int k = k0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (k < g.Kp) {
#pragma unroll
                for (int j = 0; j < 16; j++) atomicAdd(dWt + (size_t)k * N + c0 + j, v[j]);
            }
        }
    } else if (!ok && tid == 0) {
        atomicOr(status, STATUS_SPIN_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tm, tc::tmem_cols(N));
}

// ---- the network's other layers (elementwise, fp32 math on bf16 data) ----

__device__ __forceinline__ float bf(const bf16 v) { return __bfloat162float(v); }

// db[c] += sum over pixels of dY[p][dyo + c].
__global__ void k_bias_grad(const bf16* __restrict__ dY, int dys, int dyo, int C, int P, float* __restrict__ db) {
    const int c = threadIdx.x;  // blockDim.x = C (<= 256)
    float acc = 0.0f;
    for (int p = blockIdx.x; p < P; p += gridDim.x) acc += bf(dY[(size_t)p * dys + dyo + c]);
    if (c < C) atomicAdd(db + c, acc);
}

// The elementwise layers move 8 channels (one 16-byte vector) per thread;
// every channel count, pitch and offset is a multiple of 8.
union V8 {
    uint4 u;
    __nv_bfloat162 h[4];
};

__device__ __forceinline__ void unpack8(const uint4 u, float* f) {
    V8 v;
    v.u = u;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __bfloat1622float2(v.h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}

__device__ __forceinline__ uint4 pack8(const float* f) {
    return make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                      pack_bf16x2(f[6], f[7]));
}

__device__ __forceinline__ uint4 ld8(const bf16* p) { return *(const uint4*)p; }
__device__ __forceinline__ void st8(bf16* p, uint4 v) { *(uint4*)p = v; }

// dY *= (Y > 0): ReLU's gradient through its output.
__global__ void k_relu_bwd(const bf16* __restrict__ Y, int ys, int yo, bf16* dY, int dys, int dyo, int C, int P) {
    const int cv = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * cv) return;
    const int p = i / cv, c = (i - p * cv) * 8;
    float y[8], d[8];
    unpack8(ld8(Y + (size_t)p * ys + yo + c), y);
    bf16* dp = dY + (size_t)p * dys + dyo + c;
    unpack8(ld8(dp), d);
#pragma unroll
    for (int j = 0; j < 8; j++)
        if (!(y[j] > 0.0f)) d[j] = 0.0f;
    st8(dp, pack8(d));
}

// 2x2 average pool: X (B, H, W, pitch xs, offset xo) -> Y (B, H/2, W/2, C contiguous).
__global__ void k_pool_fwd(const bf16* __restrict__ X, int xs, int xo, int C, int B, int H, int W, bf16* __restrict__ Y) {
    const int h = H / 2, w = W / 2, cv = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * h * w * cv) return;
    const int q = i / cv, c = (i - q * cv) * 8;
    const int x = q % w, y = (q / w) % h, b = q / (w * h);
    const size_t p00 = (size_t)(b * H + 2 * y) * W + 2 * x;
    float s[8], t[8];
    unpack8(ld8(X + p00 * xs + xo + c), s);
    unpack8(ld8(X + (p00 + 1) * xs + xo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(ld8(X + (p00 + W) * xs + xo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(ld8(X + (p00 + W + 1) * xs + xo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] = 0.25f * (s[j] + t[j]);
    st8(Y + (size_t)q * C + c, pack8(s));
}

// Its gradient, added into dX (B, H, W, pitch dxs, offset dxo).
__global__ void k_pool_bwd(const bf16* __restrict__ dY, int C, int B, int H, int W, bf16* dX, int dxs, int dxo) {
    const int cv = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * H * W * cv) return;
    const int p = i / cv, c = (i - p * cv) * 8;
    const int x = p % W, y = (p / W) % H, b = p / (W * H);
    float g[8], d[8];
    unpack8(ld8(dY + ((size_t)(b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c), g);
    bf16* dp = dX + (size_t)p * dxs + dxo + c;
    unpack8(ld8(dp), d);
#pragma unroll
    for (int j = 0; j < 8; j++) d[j] += 0.25f * g[j];
    st8(dp, pack8(d));
}

// Nearest 2x upsample: X (B, H/2, W/2, C contiguous) -> Y (B, H, W, pitch ys, offset yo).
__global__ void k_up_fwd(const bf16* __restrict__ X, int C, int B, int H, int W, bf16* __restrict__ Y, int ys, int yo) {
    const int cv = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * H * W * cv) return;
    const int p = i / cv, c = (i - p * cv) * 8;
    const int x = p % W, y = (p / W) % H, b = p / (W * H);
    st8(Y + (size_t)p * ys + yo + c, ld8(X + ((size_t)(b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c));
}

// Its gradient: dX (B, H/2, W/2, C contiguous) = sum of the 4 children.
__global__ void k_up_bwd(const bf16* __restrict__ dY, int dys, int dyo, int C, int B, int H, int W, bf16* __restrict__ dX) {
    const int h = H / 2, w = W / 2, cv = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * h * w * cv) return;
    const int q = i / cv, c = (i - q * cv) * 8;
    const int x = q % w, y = (q / w) % h, b = q / (w * h);
    const size_t p00 = (size_t)(b * H + 2 * y) * W + 2 * x;
    float s[8], t[8];
    unpack8(ld8(dY + p00 * dys + dyo + c), s);
    unpack8(ld8(dY + (p00 + 1) * dys + dyo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(ld8(dY + (p00 + W) * dys + dyo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    unpack8(ld8(dY + (p00 + W + 1) * dys + dyo + c), t);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] += t[j];
    st8(dX + (size_t)q * C + c, pack8(s));
}

// W2[ci][(8 - tap) * cout + co] = W[co][tap * cin + ci]: the weights of the
// data-gradient convolution (a 3x3 convolution of dY).
__global__ void k_flip(const bf16* __restrict__ W, int cout, int cin, int Kp, bf16* __restrict__ W2, int Kp2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)cin * Kp2) return;
    const int ci = (int)(i / Kp2), k2 = (int)(i - (size_t)ci * Kp2);
    float v = 0.0f;
    if (k2 < 9 * cout) {
        const int tap2 = k2 / cout, co = k2 - tap2 * cout;
        v = bf(W[(size_t)co * Kp + (8 - tap2) * cin + ci]);
    }
    W2[i] = __float2bfloat16(v);
}

// Kernel prediction on demodulated radiance. Per pixel the softmax of
// logits 0..24 weights the 5 x 5 neighbourhood (clamped to the valid h x w
// image) of the irradiance irr = radiance / albedo', and the result is
// remodulated: out = albedo' * sum_t w_t irr[nb_t]. Logit 25 is the
// network's estimate e of log(relative error + 1e-3) at the pixel; `err`
// receives exp(e) - 1e-3. With `ref`, adds to *loss the mean over valid
// pixels and channels of (out - ref)^2 / (ref^2 + 0.01) and writes the
// gradient of that loss plus err_weight * mean (e - log(rel_p + 1e-3))^2
// (rel_p the pixel's own relative error, held constant) to dlogits (bf16,
// pitch 32; zero on padding pixels and on logits 26..31).
// Buffers are [B][Hp][Wp] x channels; pixels with y >= h or x >= w are padding.
__global__ void __launch_bounds__(256) k_kpn(const float* __restrict__ logits, const float* __restrict__ irr,
                                             const float* __restrict__ alb, const float* __restrict__ ref, int B,
                                             int Hp, int Wp, int h, int w, float* __restrict__ out,
                                             float* __restrict__ err, bf16* __restrict__ dlogits, float* loss,
                                             float scale, float err_weight) {
    // The 20 x 20 clamped neighbourhood of this block's 16 x 16 pixels.
    __shared__ float tile[20][20][3];
    const int bx = blockIdx.x * 16, by = blockIdx.y * 16, b = blockIdx.z;
    for (int k = threadIdx.x; k < 400; k += 256) {
        const int ly = k / 20, lx = k - ly * 20;
        const int yy = min(max(by + ly - 2, 0), h - 1), xx = min(max(bx + lx - 2, 0), w - 1);
        const float* q = irr + ((size_t)(b * Hp + yy) * Wp + xx) * 3;
        tile[ly][lx][0] = q[0];
        tile[ly][lx][1] = q[1];
        tile[ly][lx][2] = q[2];
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int x = bx + tx, y = by + ty;
    const bool inside = x < Wp && y < Hp;
    const size_t p = ((size_t)b * Hp + y) * Wp + x;
    float lsum = 0.0f;
    if (inside) {
        const bool valid = y < h && x < w;
        if (!valid) {
            if (out)
                for (int c = 0; c < 3; c++) out[p * 3 + c] = 0.0f;
            if (err) err[p] = 0.0f;
            if (ref && dlogits)
                for (int t = 0; t < 32; t++) dlogits[p * 32 + t] = __float2bfloat16(0.0f);
        } else {
            float wt[25], mx = -3.0e38f;
            const float4* lg = (const float4*)(logits + p * 32);
            float e = 0.0f;
#pragma unroll
            for (int q = 0; q < 7; q++) {
                const float4 v = __ldg(lg + q);
                const float f[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int t = 4 * q + j;
                    if (t < 25) {
                        wt[t] = f[j];
                        mx = fmaxf(mx, f[j]);
                    } else if (t == 25) {
                        e = f[j];
                    }
                }
            }
            float z = 0.0f;
#pragma unroll
            for (int t = 0; t < 25; t++) {
                wt[t] = pm_exp(wt[t] - mx);
                z += wt[t];
            }
            const float iz = 1.0f / z;
            float sm[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int t = 0; t < 25; t++) {
                wt[t] *= iz;
                const float* nb = tile[ty + t / 5][tx + t % 5];
#pragma unroll
                for (int c = 0; c < 3; c++) sm[c] += wt[t] * nb[c];
            }
            float a[3], o[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                a[c] = alb[p * 3 + c];
                o[c] = a[c] * sm[c];
            }
            if (out)
                for (int c = 0; c < 3; c++) out[p * 3 + c] = o[c];
            if (err) err[p] = fmaxf(pm_exp(e) - 1.0e-3f, 0.0f);
            if (ref) {
                float go[3], rel = 0.0f;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float r = ref[p * 3 + c], d = o[c] - r, den = r * r + 0.01f;
                    rel += d * d / den;
                    go[c] = 2.0f * d / den * scale * a[c];
                }
                lsum = rel;
                const float target = pm_log2(rel * (1.0f / 3.0f) + 1.0e-3f) * 0.693147182f;
                const float ge = 2.0f * err_weight * (e - target) * (3.0f * scale);
                float gw[25], dot = 0.0f;
#pragma unroll
                for (int t = 0; t < 25; t++) {
                    const float* nb = tile[ty + t / 5][tx + t % 5];
                    gw[t] = go[0] * nb[0] + go[1] * nb[1] + go[2] * nb[2];
                    dot += wt[t] * gw[t];
                }
                if (dlogits) {
                    bf16* d = dlogits + p * 32;
#pragma unroll
                    for (int t = 0; t < 25; t++) d[t] = __float2bfloat16(wt[t] * (gw[t] - dot));
                    d[25] = __float2bfloat16(ge);
#pragma unroll
                    for (int t = 26; t < 32; t++) d[t] = __float2bfloat16(0.0f);
                }
            }
        }
    }
    if (ref && loss) {
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum * scale);
    }
}

// Adam on a weight matrix held [rows][Kp] whose gradient is [Kp][rows]
// (transposed), or on a plain vector (gt == false). Writes the bf16 copy.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       bf16* __restrict__ wb, int rows, int Kp, int K, bool gt, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)rows * Kp) return;
    const int r = (int)(i / Kp), k = (int)(i - (size_t)r * Kp);
    if (k >= K) {
        if (wb) wb[i] = __float2bfloat16(0.0f);
        return;
    }
    const float gr = gt ? g[(size_t)k * rows + r] : g[i];
    const float mm = b1 * m[i] + (1.0f - b1) * gr;
    const float vv = b2 * v[i] + (1.0f - b2) * gr * gr;
    m[i] = mm;
    v[i] = vv;
    const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    const float nw = w[i] - upd;
    w[i] = nw;
    if (wb) wb[i] = __float2bfloat16(nw);
}

__device__ __forceinline__ float finite_or_zero(float v) { return isfinite(v) ? v : 0.0f; }

// Network inputs from a traced image (px planes, src/trace/read.rs:37-56).
// The a-trous Denoise's first-round firefly clamp (denoise.wgsl:47-134, the
// rule k_round<FIRST> applies) on B padded images of irradiance (fp32 x 3 a
// pixel): a pixel inside the h x w image whose luma exceeds 1.5 x the
// brightest of its in-image 8-neighbours + 0.05 takes those neighbours'
// mean; every other pixel is copied. Luma and the mean are summed in the
// order k_round sums them.
__global__ void k_firefly(const float* __restrict__ irr, float* __restrict__ out, int B, int Hp, int Wp, int h,
                          int w) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)B * Hp * Wp) return;
    const int x = (int)(q % (size_t)Wp), y = (int)((q / (size_t)Wp) % (size_t)Hp);
    const size_t img = q - (size_t)y * Wp - x;  // first pixel of this image
    float r = __ldg(irr + 3 * q), g = __ldg(irr + 3 * q + 1), b = __ldg(irr + 3 * q + 2);
    if (x < w && y < h) {
        float top = 0.0f, sr = 0.0f, sg = 0.0f, sb = 0.0f, nn = 0.0f;
        for (int dy = -1; dy <= 1; dy++) {
            for (int dx = -1; dx <= 1; dx++) {
                const int sx = x + dx, sy = y + dy;
                if ((dx == 0 && dy == 0) || sx < 0 || sy < 0 || sx >= w || sy >= h) continue;
                const float* c = irr + 3 * (img + (size_t)sy * Wp + sx);
                const float cr = __ldg(c), cg = __ldg(c + 1), cb = __ldg(c + 2);
                top = fmaxf(top, cr * 0.2126f + cg * 0.7152f + cb * 0.0722f);
                sr += cr;
                sg += cg;
                sb += cb;
                nn += 1.0f;
            }
        }
        if (nn > 0.0f && r * 0.2126f + g * 0.7152f + b * 0.0722f > 1.5f * top + 0.05f) {
            r = sr / nn;
            g = sg / nn;
            b = sb / nn;
        }
    }
    out[3 * q] = r;
    out[3 * q + 1] = g;
    out[3 * q + 2] = b;
}

// Per pixel of the padded image (Hp x Wp; padding pixels all zero) 16 bf16
// channels: log(1 + |irr_a - irr_b| / 2) 3, log(1 + irradiance) 3, albedo 3,
// normal 3, depth / (1 + |depth|), the fraction of samples that met
// something, log2(samples) / 8, and 1 where the first channels hold a
// spread, 0 where they do not. Radiance is the mean over the samples that
// met something (util.wgsl's emit: light sum / max(k - gone, 1)); albedo' = max(albedo,
// 0.05) per channel; irradiance = radiance / albedo'. irr_a / irr_b are the
// irradiances of the samples before and after `half` (a snapshot of the
// sums and met-sample count taken part way, phx_nn_snapshot; NULL: none) —
// their difference is the pixel's own sample spread. A plane value that is
// not finite reads as 0. Also writes irr and albedo' (fp32 x 3 each), the
// planes the predicted kernels filter and remodulate.
__global__ void k_features(const uint32_t* __restrict__ px, const float4* __restrict__ half, int w, int h, int Hp,
                           int Wp, bf16* __restrict__ feat, float* __restrict__ irr, float* __restrict__ alb) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Hp * Wp) return;
    const int x = q % Wp, y = q / Wp;
    float f[16];
#pragma unroll
    for (int j = 0; j < 16; j++) f[j] = 0.0f;
    float ir[3] = {0.0f, 0.0f, 0.0f}, ad[3] = {0.0f, 0.0f, 0.0f};
    if (x < w && y < h) {
        const size_t n = (size_t)w * h, i = (size_t)y * w + x;
        const uint32_t cnt = px[31 * n + i];
        const float k = (float)max(cnt, 1u);
        const float gone = __uint_as_float(px[33 * n + i]);
        const float met = fmaxf(k - gone, 1.0f);
        const float ln2 = 0.693147182f;
        float4 hs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (half) hs = half[i];
        const float met_total = (float)cnt - gone;
        const bool spread = half && hs.w >= 1.0f && met_total - hs.w >= 1.0f;
        const float hsum[3] = {hs.x, hs.y, hs.z};
        float nn = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            // a sample that overflowed (or a NaN) gives no input rather than a poisoned one
            const float sum = __uint_as_float(px[n + 3 * i + c]);
            const float rad = finite_or_zero(fmaxf(sum / met, 0.0f));
            const float al = finite_or_zero(__uint_as_float(px[7 * n + 3 * i + c]) / k);
            ad[c] = fmaxf(al, 0.05f);
            ir[c] = rad / ad[c];
            if (spread) {
                const float ra = fmaxf(hsum[c] / hs.w, 0.0f);
                const float rb = fmaxf((sum - hsum[c]) / (met_total - hs.w), 0.0f);
                f[c] = pm_log2(1.0f + finite_or_zero(fabsf(ra - rb) * 0.5f / ad[c])) * ln2;
            }
            f[3 + c] = pm_log2(1.0f + ir[c]) * ln2;
            f[6 + c] = al;
            f[9 + c] = finite_or_zero(__uint_as_float(px[10 * n + 3 * i + c]));
            nn += f[9 + c] * f[9 + c];
        }
        const float inv = nn > 0.0f ? 1.0f / sqrtf(nn) : 0.0f;
#pragma unroll
        for (int c = 0; c < 3; c++) f[9 + c] *= inv;
        const float d = finite_or_zero(__uint_as_float(px[13 * n + i]) / k);
        f[12] = d / (1.0f + fabsf(d));
        f[13] = fmaxf(1.0f - gone / k, 0.0f);
        f[14] = pm_log2(k) * 0.125f;
        f[15] = spread ? 1.0f : 0.0f;
    }
    uint4* o = (uint4*)(feat + (size_t)q * 16);
    o[0] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7]));
    o[1] = make_uint4(pack_bf16x2(f[8], f[9]), pack_bf16x2(f[10], f[11]), pack_bf16x2(f[12], f[13]),
                      pack_bf16x2(f[14], f[15]));
#pragma unroll
    for (int c = 0; c < 3; c++) {
        irr[(size_t)q * 3 + c] = ir[c];
        alb[(size_t)q * 3 + c] = ad[c];
    }
}

// The sums and met-sample count of a px image now: the `half` snapshot of
// k_features (float4 per pixel: linear sums xyz, samples - missed).
__global__ void k_snapshot(const uint32_t* __restrict__ px, uint32_t n, float4* __restrict__ snap) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    snap[i] = make_float4(__uint_as_float(px[n + 3 * i]), __uint_as_float(px[n + 3 * i + 1]),
                          __uint_as_float(px[n + 3 * i + 2]),
                          (float)px[31 * (size_t)n + i] - __uint_as_float(px[33 * (size_t)n + i]));
}

// Mean of the per-pixel error estimate over each ts x ts tile of the valid
// image (one block per tile); counts the tiles above `threshold`.
__global__ void k_tile_err(const float* __restrict__ err, int w, int h, int Wp, int ts, float threshold,
                           float* __restrict__ tile_err, uint32_t* fallback) {
    const int tx = blockIdx.x, ty = blockIdx.y;
    const int x0 = tx * ts, y0 = ty * ts;
    const int tw = min(ts, w - x0), th = min(ts, h - y0);
    float s = 0.0f;
    for (int j = threadIdx.x; j < tw * th; j += blockDim.x) {
        const int yy = y0 + j / tw, xx = x0 + j % tw;
        s += err[(size_t)yy * Wp + xx];
    }
    __shared__ float part[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) t += part[j];
        t /= (float)(tw * th);
        tile_err[ty * gridDim.x + tx] = t;
        if (!(t <= threshold)) atomicAdd(fallback, 1u);
    }
}

// Writes the learned result into the px planes for every pixel whose tile
// estimate is within `threshold` (the rest keep what Denoise wrote):
// the scene-linear sums so that their mean over the samples that met
// something (emit's light sum / max(k - gone, 1)) is `out` (unless
// keep), the shown value and the packed display pixel, as the last Denoise
// round does (denoise.wgsl, Standard view transform).
__global__ void k_compose(const float* __restrict__ out, const float* __restrict__ tile_err, int w, int h, int Wp,
                          int ts, float threshold, int keep, float exposure, float gamma, uint32_t* __restrict__ px) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int tiles_x = (w + ts - 1) / ts;
    if (!(tile_err[(y / ts) * tiles_x + x / ts] <= threshold)) return;
    const uint32_t n = (uint32_t)w * h, i = (uint32_t)y * w + x;
    const uint32_t cnt = px[31 * n + i];
    const float k = 1.0f / (float)(cnt > 1 ? cnt : 1);
    const float gone = __uint_as_float(px[33 * n + i]);
    const float met = 1.0f - gone * k;
    const size_t q = (size_t)y * Wp + x;
    f3 lin = mk(out[q * 3], out[q * 3 + 1], out[q * 3 + 2]);
    if (!(met > 0.5f * k)) lin = mk(0.0f);
    if (!keep) {
        const float m = fmaxf((float)(cnt > 1 ? cnt : 1) - gone, 1.0f);
        px[n + 3 * i] = __float_as_uint(lin.x * m);
        px[n + 3 * i + 1] = __float_as_uint(lin.y * m);
        px[n + 3 * i + 2] = __float_as_uint(lin.z * m);
    }
    const float cov = __uint_as_float(px[23 * n + i]) * k;
    const f3 grid = mk(__uint_as_float(px[20 * n + 3 * i]), __uint_as_float(px[20 * n + 3 * i + 1]),
                       __uint_as_float(px[20 * n + 3 * i + 2])) * k;
    const f3 shown = view_transform_std(lin, exposure, gamma) * (1.0f - cov) + grid;
    px[4 * n + 3 * i] = __float_as_uint(shown.x);
    px[4 * n + 3 * i + 1] = __float_as_uint(shown.y);
    px[4 * n + 3 * i + 2] = __float_as_uint(shown.z);
    px[i] = pack_rgba(shown, __uint_as_float(px[24 * n + i]) * k);
}

template <int N, int CC, int T, bool RELU, bool F32>
int32_t conv_fwd_n(Ctx* c, const bf16* X, const bf16* W, const float* bias, void* Y, const Geo& g) {
    const int smem = Conv<N, CC, T>::TOTAL;
    static std::atomic<uint64_t> done{0};
    PHX_TRY(smem_limit(k_conv_fwd<N, CC, T, RELU, F32>, smem, c->device, done));
    const uint32_t blocks = (uint32_t)g.B * ((g.H + TY - 1) / TY) * ((g.W + TX * T - 1) / (TX * T));
    k_conv_fwd<N, CC, T, RELU, F32><<<blocks, 128, smem, c->stream>>>(X, W, bias, Y, g, c->status);
    return cuda_check(cudaGetLastError(), "conv fwd");
}

constexpr size_t WS_MAX_SMEM = 110 * 1024;

template <int N, bool RELU, bool F32>
int32_t conv_ws_n(Ctx* c, const bf16* X, const bf16* W, const float* bias, void* Y, const Geo& g) {
    const int smem = (int)ConvWS<N>::bytes(g.cin);
    static std::atomic<uint64_t> done{0};
    PHX_TRY(smem_limit(k_conv_ws<N, RELU, F32>, (int)WS_MAX_SMEM, c->device, done));
    // Blocks per SM: by shared memory (the SM's 228 KB less 1 KB per block,
    // this kernel's 1 KB of static data), by the 512 TMEM columns (two
    // accumulators a block) and by threads.
    const int by_smem = (228 * 1024) / (smem + 2 * 1024);
    const int by_tmem = (int)(512 / (2 * tc::tmem_cols(N)));
    const int per_sm = std::max(1, std::min(std::min(by_smem, by_tmem), 16));
    const int ntiles = g.B * ((g.H + TY - 1) / TY) * ((g.W + TX - 1) / TX);
    const int grid = std::min(ntiles, per_sm * c->sms);
    k_conv_ws<N, RELU, F32><<<grid, 128, smem, c->stream>>>(X, W, bias, Y, g, c->status);
    return cuda_check(cudaGetLastError(), "conv fwd (weight-stationary)");
}

// The head (32 outputs, no ReLU) with the kernel-prediction epilogue.
int32_t conv_kpn(Ctx* c, const bf16* X, const bf16* W, const float* bias, const Geo& g, const KpnOut& kp) {
    const int smem = (int)ConvWS<32>::bytes(g.cin);
    if ((size_t)smem > WS_MAX_SMEM) return fail(PHX_ERR_INVALID, "conv+kpn: %d input channels do not fit", g.cin);
    static std::atomic<uint64_t> done{0};
    PHX_TRY(smem_limit(k_conv_ws<32, false, true, true>, (int)WS_MAX_SMEM, c->device, done));
    const int by_smem = (228 * 1024) / (smem + 2 * 1024);
    const int per_sm = std::max(1, std::min(std::min(by_smem, (int)(512 / (2 * tc::tmem_cols(32)))), 16));
    const int ntiles = g.B * ((g.H + TY - 1) / TY) * ((g.W + TX - 1) / TX);
    const int grid = std::min(ntiles, per_sm * c->sms);
    k_conv_ws<32, false, true, true><<<grid, 128, smem, c->stream>>>(X, W, bias, nullptr, g, c->status, kp);
    return cuda_check(cudaGetLastError(), "conv + kpn");
}

// The weight-stationary form where two of its blocks fit an SM, else the
// chunked form over 16 channels a chunk.
template <int N, bool RELU, bool F32>
int32_t conv_fwd_cc(Ctx* c, const bf16* X, const bf16* W, const float* bias, void* Y, const Geo& g) {
    if (N <= 128 && ConvWS<N>::bytes(g.cin) <= WS_MAX_SMEM) return conv_ws_n<N, RELU, F32>(c, X, W, bias, Y, g);
    // chunked: several tiles a block where N is small (their weights read once)
    constexpr int T = N <= 32 ? 4 : (N <= 64 ? 2 : 1);
    return conv_fwd_n<N, 16, T, RELU, F32>(c, X, W, bias, Y, g);
}

template <bool RELU, bool F32>
int32_t conv_fwd_any(Ctx* c, const bf16* X, const bf16* W, const float* bias, void* Y, const Geo& g) {
    switch (g.cout) {
        case 32: return conv_fwd_cc<32, RELU, F32>(c, X, W, bias, Y, g);
        case 64: return conv_fwd_cc<64, RELU, F32>(c, X, W, bias, Y, g);
        case 96: return conv_fwd_cc<96, RELU, F32>(c, X, W, bias, Y, g);
        case 128: return conv_fwd_cc<128, RELU, F32>(c, X, W, bias, Y, g);
        case 160: return conv_fwd_cc<160, RELU, F32>(c, X, W, bias, Y, g);
    }
    return fail(PHX_ERR_INVALID, "conv: output tile of %d channels (32, 64, 96, 128 or 160)", g.cout);
}

template <int N>
int32_t wgrad_n(Ctx* c, const bf16* X, const bf16* dY, int dys, int dyo, float* dWt, const Geo& g) {
    const int smem = Plan<N>::TOTAL;
    static std::atomic<uint64_t> done{0};
    PHX_TRY(smem_limit(k_conv_wgrad<N>, smem, c->device, done));
    const int P = g.B * g.H * g.W;
    // Split the pixel reduction so the grid covers the SMs a few times.
    const int kblocks = (g.Kp + tc::BM - 1) / tc::BM;
    int splits = (c->sms * 2 + kblocks - 1) / kblocks;
    int chunk = (P + splits - 1) / splits;
    chunk = (chunk + tc::BK - 1) / tc::BK * tc::BK;
    splits = (P + chunk - 1) / chunk;
    k_conv_wgrad<N><<<dim3(kblocks, splits), 128, smem, c->stream>>>(X, dY, dys, dyo, dWt, g, chunk, c->status);
    return cuda_check(cudaGetLastError(), "conv wgrad");
}

int32_t check_geo(const Geo& g) {
    if (g.B <= 0 || g.H <= 0 || g.W <= 0) return fail(PHX_ERR_INVALID, "conv: empty image");
    if (g.cin % 16 || g.xs % 8 || g.xo % 8 || g.ys % 8 || g.yo % 8)
        return fail(PHX_ERR_INVALID, "conv: cin a multiple of 16, pitches and offsets multiples of 8");
    if (g.Kp % 64 || g.Kp < g.K) return fail(PHX_ERR_INVALID, "conv: Kp %d must cover K %d in steps of 64", g.Kp, g.K);
    if (g.xo < 0 || g.xo + g.cin > g.xs || g.yo < 0 || g.yo + g.cout > g.ys)
        return fail(PHX_ERR_INVALID, "conv: channel window outside the pixel pitch");
    return PHX_OK;
}

uint32_t blocks_for(size_t n) { return (uint32_t)((n + 255) / 256); }

}  // namespace
}  // namespace phx

using namespace phx;

extern "C" {

int32_t phx_nn_conv_fwd(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* W, int32_t Kp,
                        const float* bias, void* Y, int32_t ys, int32_t yo, int32_t cout, int32_t B, int32_t H,
                        int32_t Wd, int32_t relu, int32_t out_f32) {
    if (!ctx || !X || !W || !bias || !Y) return fail(PHX_ERR_INVALID, "null argument");
    Geo g{B, H, Wd, cin, xs, xo, cout, ys, yo, 9 * cin, Kp};
    PHX_TRY(check_geo(g));
    PHX_TRY(use(&ctx->c));
    const bf16* x = (const bf16*)X;
    const bf16* w = (const bf16*)W;
    if (out_f32) return relu ? conv_fwd_any<true, true>(&ctx->c, x, w, bias, Y, g)
                             : conv_fwd_any<false, true>(&ctx->c, x, w, bias, Y, g);
    return relu ? conv_fwd_any<true, false>(&ctx->c, x, w, bias, Y, g) : conv_fwd_any<false, false>(&ctx->c, x, w, bias, Y, g);
}

int32_t phx_nn_conv_kpn(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* W, int32_t Kp,
                        const float* bias, const float* irr, const float* alb, int32_t B, int32_t Hp, int32_t Wp,
                        int32_t h, int32_t w, float* out, float* err) {
    if (!ctx || !X || !W || !bias || !irr || !alb || !out || !err) return fail(PHX_ERR_INVALID, "null argument");
    if (h <= 0 || w <= 0 || h > Hp || w > Wp) return fail(PHX_ERR_INVALID, "conv+kpn: bad valid region");
    Geo g{B, Hp, Wp, cin, xs, xo, 32, 32, 0, 9 * cin, Kp};
    PHX_TRY(check_geo(g));
    PHX_TRY(use(&ctx->c));
    return conv_kpn(&ctx->c, (const bf16*)X, (const bf16*)W, bias, g, KpnOut{irr, alb, out, err, h, w});
}

int32_t phx_nn_conv_wgrad(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t cin, const void* dY,
                          int32_t dys, int32_t dyo, int32_t cout, float* dWt, int32_t Kp, int32_t B, int32_t H,
                          int32_t Wd) {
    if (!ctx || !X || !dY || !dWt) return fail(PHX_ERR_INVALID, "null argument");
    Geo g{B, H, Wd, cin, xs, xo, cout, cout, 0, 9 * cin, Kp};
    PHX_TRY(check_geo(g));
    if (dys % 8 || dyo % 8 || dyo < 0 || dyo + cout > dys)
        return fail(PHX_ERR_INVALID, "wgrad: dY pitch/offset must be multiples of 8 holding cout channels");
    PHX_TRY(use(&ctx->c));
    const bf16* x = (const bf16*)X;
    const bf16* d = (const bf16*)dY;
    switch (cout) {
        case 32: return wgrad_n<32>(&ctx->c, x, d, dys, dyo, dWt, g);
        case 64: return wgrad_n<64>(&ctx->c, x, d, dys, dyo, dWt, g);
        case 96: return wgrad_n<96>(&ctx->c, x, d, dys, dyo, dWt, g);
        case 128: return wgrad_n<128>(&ctx->c, x, d, dys, dyo, dWt, g);
        case 160: return wgrad_n<160>(&ctx->c, x, d, dys, dyo, dWt, g);
    }
    return fail(PHX_ERR_INVALID, "wgrad: %d output channels (32, 64, 96, 128 or 160)", cout);
}

int32_t phx_nn_bias_grad(phx_ctx ctx, const void* dY, int32_t dys, int32_t dyo, int32_t C, int32_t P, float* db) {
    if (!ctx || !dY || !db || C <= 0 || C > 256 || P < 0 || dyo < 0 || dyo + C > dys)
        return fail(PHX_ERR_INVALID, "bias grad arguments");
    if (P == 0) return PHX_OK;
    PHX_TRY(use(&ctx->c));
    k_bias_grad<<<std::min(P, 1024), C, 0, ctx->c.stream>>>((const bf16*)dY, dys, dyo, C, P, db);
    return cuda_check(cudaGetLastError(), "bias grad");
}

int32_t phx_nn_relu_bwd(phx_ctx ctx, const void* Y, int32_t ys, int32_t yo, void* dY, int32_t dys, int32_t dyo,
                        int32_t C, int32_t P) {
    if (!ctx || !Y || !dY || C <= 0 || C % 8 || P <= 0 || yo < 0 || yo + C > ys || dyo < 0 || dyo + C > dys ||
        (ys | yo | dys | dyo) % 8)
        return fail(PHX_ERR_INVALID, "relu bwd arguments");
    PHX_TRY(use(&ctx->c));
    k_relu_bwd<<<blocks_for((size_t)P * (C / 8)), 256, 0, ctx->c.stream>>>((const bf16*)Y, ys, yo, (bf16*)dY, dys, dyo, C, P);
    return cuda_check(cudaGetLastError(), "relu bwd");
}

int32_t phx_nn_pool_fwd(phx_ctx ctx, const void* X, int32_t xs, int32_t xo, int32_t C, int32_t B, int32_t H, int32_t W,
                        void* Y) {
    if (!ctx || !X || !Y || B <= 0 || H <= 0 || W <= 0 || C <= 0 || C % 8 || H % 2 || W % 2 || xo < 0 ||
        xo + C > xs || (xs | xo) % 8)
        return fail(PHX_ERR_INVALID, "pool arguments");
    PHX_TRY(use(&ctx->c));
    k_pool_fwd<<<blocks_for((size_t)B * (H / 2) * (W / 2) * (C / 8)), 256, 0, ctx->c.stream>>>((const bf16*)X, xs, xo, C, B, H,
                                                                                        W, (bf16*)Y);
    return cuda_check(cudaGetLastError(), "pool fwd");
}

int32_t phx_nn_pool_bwd(phx_ctx ctx, const void* dY, int32_t C, int32_t B, int32_t H, int32_t W, void* dX, int32_t dxs,
                        int32_t dxo) {
    if (!ctx || !dY || !dX || B <= 0 || H <= 0 || W <= 0 || C <= 0 || C % 8 || H % 2 || W % 2 || dxo < 0 ||
        dxo + C > dxs || (dxs | dxo) % 8)
        return fail(PHX_ERR_INVALID, "pool arguments");
    PHX_TRY(use(&ctx->c));
    k_pool_bwd<<<blocks_for((size_t)B * H * W * (C / 8)), 256, 0, ctx->c.stream>>>((const bf16*)dY, C, B, H, W, (bf16*)dX, dxs,
                                                                              dxo);
    return cuda_check(cudaGetLastError(), "pool bwd");
}

int32_t phx_nn_up_fwd(phx_ctx ctx, const void* X, int32_t C, int32_t B, int32_t H, int32_t W, void* Y, int32_t ys,
                      int32_t yo) {
    if (!ctx || !X || !Y || B <= 0 || H <= 0 || W <= 0 || C <= 0 || C % 8 || H % 2 || W % 2 || yo < 0 ||
        yo + C > ys || (ys | yo) % 8)
        return fail(PHX_ERR_INVALID, "upsample arguments");
    PHX_TRY(use(&ctx->c));
    k_up_fwd<<<blocks_for((size_t)B * H * W * (C / 8)), 256, 0, ctx->c.stream>>>((const bf16*)X, C, B, H, W, (bf16*)Y, ys, yo);
    return cuda_check(cudaGetLastError(), "up fwd");
}

int32_t phx_nn_up_bwd(phx_ctx ctx, const void* dY, int32_t dys, int32_t dyo, int32_t C, int32_t B, int32_t H, int32_t W,
                      void* dX) {
    if (!ctx || !dY || !dX || B <= 0 || H <= 0 || W <= 0 || C <= 0 || C % 8 || H % 2 || W % 2 || dyo < 0 ||
        dyo + C > dys || (dys | dyo) % 8)
        return fail(PHX_ERR_INVALID, "upsample arguments");
    PHX_TRY(use(&ctx->c));
    k_up_bwd<<<blocks_for((size_t)B * (H / 2) * (W / 2) * (C / 8)), 256, 0, ctx->c.stream>>>((const bf16*)dY, dys, dyo, C, B,
                                                                                      H, W, (bf16*)dX);
    return cuda_check(cudaGetLastError(), "up bwd");
}

int32_t phx_nn_flip(phx_ctx ctx, const void* W, int32_t cout, int32_t cin, int32_t Kp, void* W2, int32_t Kp2) {
    if (!ctx || !W || !W2 || Kp2 < 9 * cout || Kp2 % 64) return fail(PHX_ERR_INVALID, "flip arguments");
    PHX_TRY(use(&ctx->c));
    k_flip<<<blocks_for((size_t)cin * Kp2), 256, 0, ctx->c.stream>>>((const bf16*)W, cout, cin, Kp, (bf16*)W2, Kp2);
    return cuda_check(cudaGetLastError(), "flip");
}

int32_t phx_nn_kpn(phx_ctx ctx, const float* logits, const float* irr, const float* alb, const float* ref, int32_t B,
                   int32_t Hp, int32_t Wp, int32_t h, int32_t w, float* out, float* err, void* dlogits, float* loss,
                   float err_weight) {
    if (!ctx || !logits || !irr || !alb) return fail(PHX_ERR_INVALID, "null argument");
    if (B <= 0 || h <= 0 || w <= 0 || h > Hp || w > Wp) return fail(PHX_ERR_INVALID, "kpn: bad image size");
    PHX_TRY(use(&ctx->c));
    const float scale = 1.0f / (3.0f * (float)B * (float)h * (float)w);
    const dim3 grid((Wp + 15) / 16, (Hp + 15) / 16, B);
    k_kpn<<<grid, 256, 0, ctx->c.stream>>>(logits, irr, alb, ref, B, Hp, Wp, h, w, out, err, (bf16*)dlogits, loss,
                                           scale, err_weight);
    return cuda_check(cudaGetLastError(), "kpn");
}

int32_t phx_nn_adam(phx_ctx ctx, float* w, const float* g, float* m, float* v, void* wb, int32_t rows, int32_t Kp,
                    int32_t K, int32_t g_transposed, float lr, float b1, float b2, float eps, int32_t step) {
    if (!ctx || !w || !g || !m || !v || step < 1) return fail(PHX_ERR_INVALID, "adam arguments");
    PHX_TRY(use(&ctx->c));
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<blocks_for((size_t)rows * Kp), 256, 0, ctx->c.stream>>>(w, g, m, v, (bf16*)wb, rows, Kp, K, g_transposed != 0,
                                                                    lr, b1, b2, eps, c1, c2);
    return cuda_check(cudaGetLastError(), "adam");
}

int32_t phx_nn_features(phx_ctx ctx, const uint32_t* px, const float* half, int32_t w, int32_t h, int32_t Hp,
                        int32_t Wp, void* feat, float* irr, float* alb) {
    if (!ctx || !px || !feat || !irr || !alb || w <= 0 || h <= 0 || Hp < h || Wp < w)
        return fail(PHX_ERR_INVALID, "features arguments");
    PHX_TRY(use(&ctx->c));
    k_features<<<(Hp * Wp + 255) / 256, 256, 0, ctx->c.stream>>>(px, (const float4*)half, w, h, Hp, Wp, (bf16*)feat,
                                                                 irr, alb);
    return cuda_check(cudaGetLastError(), "features");
}

int32_t phx_nn_firefly(phx_ctx ctx, const float* irr, float* out, int32_t B, int32_t Hp, int32_t Wp, int32_t h,
                       int32_t w) {
    if (!ctx || !irr || !out || irr == out || B <= 0 || h <= 0 || w <= 0 || Hp < h || Wp < w)
        return fail(PHX_ERR_INVALID, "firefly arguments");
    PHX_TRY(use(&ctx->c));
    const size_t total = (size_t)B * Hp * Wp;
    k_firefly<<<(unsigned)((total + 255) / 256), 256, 0, ctx->c.stream>>>(irr, out, B, Hp, Wp, h, w);
    return cuda_check(cudaGetLastError(), "firefly");
}

int32_t phx_nn_snapshot(phx_ctx ctx, const uint32_t* px, uint32_t w, uint32_t h, float* snap) {
    if (!ctx || !px || !snap) return fail(PHX_ERR_INVALID, "null argument");
    const uint32_t n = w * h;
    if (n == 0) return PHX_OK;
    PHX_TRY(use(&ctx->c));
    k_snapshot<<<(n + 255) / 256, 256, 0, ctx->c.stream>>>(px, n, (float4*)snap);
    return cuda_check(cudaGetLastError(), "snapshot");
}

int32_t phx_nn_compose(phx_ctx ctx, uint32_t* px, int32_t w, int32_t h, int32_t Wp, const float* out, const float* err,
                       int32_t tile, float threshold, int32_t keep, float exposure, float gamma, float* tile_err,
                       uint32_t* fallback) {
    if (!ctx || !px || !out || !err || !tile_err || !fallback || tile <= 0 || w <= 0 || h <= 0 || Wp < w)
        return fail(PHX_ERR_INVALID, "compose arguments");
    PHX_TRY(use(&ctx->c));
    const dim3 tiles((w + tile - 1) / tile, (h + tile - 1) / tile);
    PHX_CUDA(cudaMemsetAsync(fallback, 0, sizeof(uint32_t), ctx->c.stream));
    k_tile_err<<<tiles, 256, 0, ctx->c.stream>>>(err, w, h, Wp, tile, threshold, tile_err, fallback);
    PHX_CUDA(cudaGetLastError());
    const dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    k_compose<<<grid, block, 0, ctx->c.stream>>>(out, tile_err, w, h, Wp, tile, threshold, keep, exposure, gamma, px);
    return cuda_check(cudaGetLastError(), "compose");
}

int32_t phx_gemm_bf16(phx_ctx ctx, const void* A, const void* B, float* D, uint32_t M, uint32_t N,
                                 uint32_t K) {
    if (!ctx || !A || !B || !D) return fail(PHX_ERR_INVALID, "null argument");
    if (M == 0 || M % 128 || K == 0 || K % 64)
        return fail(PHX_ERR_INVALID, "gemm: M %u must be a multiple of 128 and K %u of 64", M, K);
    PHX_TRY(use(&ctx->c));
    const bf16* a = (const bf16*)A;
    const bf16* b = (const bf16*)B;
    switch (N) {
        case 32: return launch_gemm<32>(&ctx->c, a, b, D, (int)M, (int)K);
        case 64: return launch_gemm<64>(&ctx->c, a, b, D, (int)M, (int)K);
        case 96: return launch_gemm<96>(&ctx->c, a, b, D, (int)M, (int)K);
        case 128: return launch_gemm<128>(&ctx->c, a, b, D, (int)M, (int)K);
        case 160: return launch_gemm<160>(&ctx->c, a, b, D, (int)M, (int)K);
    }
    return fail(PHX_ERR_INVALID, "gemm: N %u must be 32, 64, 96, 128 or 160", N);
}

}  // extern "C"
