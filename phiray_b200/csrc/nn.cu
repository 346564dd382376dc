// BF16 tensor-core kernels for the learned denoiser (tcgen05, tc.cuh).
//
// phx_gemm_bf16: D (fp32, M x N) = A (bf16, M x K, row-major) x B^T (B bf16,
// N x K, row-major). The building block the convolutions stage through; also
// the engine's own parity check against a plain matrix product.
#include <cuda_bf16.h>

#include "internal.cuh"
#include "tc.cuh"

namespace phx {
namespace {

using bf16 = __nv_bfloat16;

// Shared-memory plan of one CTA: A tile, room past it, B tile, room past it.
// The room keeps every byte the MMAs could address inside the allocation
// even if a descriptor's strides were read the other way round.
template <int N>
struct Plan {
    static constexpr int A_BYTES = tc::BM * tc::BK * 2;
    static constexpr int B_BYTES = N * tc::BK * 2;
    static constexpr int A_ROOM = 16 * 1024;
    static constexpr int B_ROOM = 64 * 1024;
    static constexpr int A_OFF = 0;
    static constexpr int B_OFF = A_BYTES + A_ROOM;
    static constexpr int TOTAL = B_OFF + B_BYTES + B_ROOM;
};

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
    PHX_CUDA(cudaFuncSetAttribute(k_gemm_bf16<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_gemm_bf16<N><<<M / tc::BM, 128, smem, c->stream>>>(A, B, D, M, K, c->status);
    return cuda_check(cudaGetLastError(), "gemm bf16");
}

}  // namespace
}  // namespace phx

using namespace phx;

extern "C" int32_t phx_gemm_bf16(phx_ctx ctx, const void* A, const void* B, float* D, uint32_t M, uint32_t N,
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
