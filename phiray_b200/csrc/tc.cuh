// A BF16 tensor-core tile engine for sm_100a: tcgen05.mma with the fp32
// accumulator in tensor memory (TMEM), operands staged in shared memory in
// the canonical K-major, no-swizzle ("interleave") layout, one elected thread
// issuing the MMAs and committing them to an mbarrier, the epilogue reading
// TMEM back with tcgen05.ld.
//
// One CTA of 128 threads (4 warps) owns a 128 x N tile of D (N a multiple of
// 16, 16..256). For each K chunk of 64 the caller's loader fills the A tile
// (128 rows x 64 k) and the B tile (N rows x 64 k); four MMAs of K = 16 are
// issued on them. Layout of a tile with R rows: 8 x 8 "core matrices" of 128
// bytes (8 rows of 16 bytes); core (row group g, k chunk c) sits at byte
// (c * R/8 + g) * 128, so one MMA's K = 16 slice is two k chunks LBO =
// R/8 * 128 bytes apart and row groups are SBO = 128 bytes apart.
//
// Descriptor bit layouts (sm100 UMMA): smem descriptor = start >> 4 (bits
// 0-13), LBO >> 4 (16-29), SBO >> 4 (32-45), version 1 (46-47), layout type
// 0 = no swizzle (61-63). Instruction descriptor for BF16 x BF16 -> F32,
// both operands K-major: c_format 1 (bits 4-5), a_format 1 (7-9), b_format 1
// (10-12), N >> 3 (17-22), M >> 4 (24-28).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace phx {
namespace tc {

constexpr int BM = 128;  // rows of a CTA tile (TMEM lanes)
constexpr int BK = 64;   // k per staged chunk (four MMAs of 16)
constexpr uint32_t WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) inside a staged tile of R rows.
__device__ __forceinline__ uint32_t tile_off(int r, int k, int R) {
    return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((start >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // version: sm100
    return d;                // layout type 0: no swizzle
}

__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__host__ __device__ constexpr uint32_t tmem_cols(int N) {
    return N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

// One arrival on an mbarrier (this thread's).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait on an mbarrier phase; false when `limit` polls ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t limit = WAIT_LIMIT) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

// D(tmem) (+)= A(smem desc) x B(smem desc)^T, one K = 16 step.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// Each thread of a warp reads 16 consecutive fp32 columns of its TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* out) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) out[j] = __uint_as_float(r[j]);
}

// Issues the four K = 16 MMAs of one staged chunk (called by one thread).
template <int N>
__device__ __forceinline__ void mma_chunk(uint32_t tmem_d, const uint8_t* a_tile, const uint8_t* b_tile, bool first) {
    constexpr uint32_t idesc = instr_desc_bf16(BM, N);
    constexpr uint32_t a_lbo = (BM / 8) * 128, b_lbo = (N / 8) * 128;
    // one descriptor per operand; each K = 16 step adds 2 * LBO / 16 to its
    // start-address field (shared-memory offsets stay below 2^18 bytes, so the
    // 14-bit field does not carry)
    const uint64_t da0 = smem_desc(smem_addr(a_tile), a_lbo, 128);
    const uint64_t db0 = smem_desc(smem_addr(b_tile), b_lbo, 128);
#pragma unroll
    for (int s = 0; s < BK / 16; s++) {
        const uint64_t da = da0 + (uint64_t)((s * 2 * a_lbo) >> 4);
        const uint64_t db = db0 + (uint64_t)((s * 2 * b_lbo) >> 4);
        mma_bf16(tmem_d, da, db, idesc, (first && s == 0) ? 0u : 1u);
    }
}

}  // namespace tc
}  // namespace phx
