// The LBVH build's device arrays and the enqueue functions that run it
// (bvh.cu), shared with the tracer, which builds its tree over face boxes.
#pragma once

#include "internal.cuh"

namespace phx {

constexpr int LBVH_TILE = 4096;  // radix-sort tile (256 threads x 16 keys)
constexpr int LBVH_PASSES = 4;   // 8-bit digits over the 30-bit Morton code

// A device-side switch on a launch: the kernel does its work only when
// *word == want (word NULL: always). A captured CUDA graph can then hold
// both a rebuild and a refit and choose per replay by one word in device
// memory, which every gated kernel reads before doing anything else.
struct Gate {
    const uint32_t* word = nullptr;
    uint32_t want = 0;
#ifdef __CUDACC__
    __device__ __forceinline__ bool off() const { return word != nullptr && *word != want; }
#endif
};

#ifdef __CUDACC__
// Decoupled look-back words of the radix sort: a tile's count for one digit
// with a flag — its own count only (AGG) or the inclusive prefix (INC).
constexpr uint32_t LOOKBACK_AGG = 1u << 30;
constexpr uint32_t LOOKBACK_INC = 2u << 30;
constexpr uint32_t LOOKBACK_VALUE = (1u << 30) - 1;

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The exclusive prefix of digit d for tile `tile` (> 0): walks back over
// the earlier tiles' words (256 per tile), adding aggregates until an
// inclusive prefix. A word not yet written is polled again, at most `limit`
// times in all; past that the wait gives up, sets STATUS_SPIN_LIMIT in
// *status and returns what it has (the caller's result is then wrong and the
// host reports the status instead of it).
__device__ __forceinline__ uint32_t lookback_prefix(const uint32_t* lookback, uint32_t tile, uint32_t d,
                                                    uint32_t limit, uint32_t* status) {
    uint32_t prefix = 0, spins = 0;
    int t = (int)tile - 1;
    while (t >= 0) {
        const uint32_t v = ld_relaxed(lookback + (size_t)t * 256 + d);
        const uint32_t flag = v & ~LOOKBACK_VALUE;
        if (flag == 0) {
            if (++spins > limit) {
                atomicOr(status, STATUS_SPIN_LIMIT);
                break;
            }
            if (spins > 32) __nanosleep(64);
            continue;
        }
        prefix += v & LOOKBACK_VALUE;
        if (flag == LOOKBACK_INC) break;
        t--;
    }
    return prefix;
}

// The climb of the atomic bottom-up refit (Bvh::refit's bounds, build.rs:
// 180-194) from node i, whose box (lx .. hz) is already stored: at each
// parent the first arriving child stops and the second unions its box with
// its sibling's (left box first) and carries on up. counters[] start even
// and every reachable inner node gets exactly two arrivals, so they need no
// reset between refits. A climb longer than any Karras tree (65 levels)
// means a corrupt parent array: STATUS_BAD_INDEX, and the climb stops.
__device__ __forceinline__ void refit_climb(uint32_t i, float lx, float ly, float lz, float hx, float hy, float hz,
                                            const uint32_t* __restrict__ parent, float4* nodes, uint32_t* counters,
                                            uint32_t* status) {
    for (int hops = 0; i != 0; hops++) {
        if (hops > 80) {
            atomicOr(status, STATUS_BAD_INDEX);
            return;
        }
        const uint32_t p = __ldg(parent + i);
        // p's child links (fixed during a refit) are read before the
        // arrival count, so the sibling is known when the count returns
        const uint32_t l = __ldcg((const uint32_t*)(nodes + 2 * (size_t)p) + 3);
        const uint32_t r = __ldcg((const uint32_t*)(nodes + 2 * (size_t)p + 1) + 3);
        __threadfence();
        const uint32_t old = atomicAdd(counters + p, 1u);
        if ((old & 1u) == 0) return;  // first child here: the sibling finishes p
        __threadfence();
        const bool is_left = (l == i);
        const uint32_t sib = is_left ? r : l;
        const float4 sa = __ldcg(nodes + 2 * (size_t)sib), sb = __ldcg(nodes + 2 * (size_t)sib + 1);
        if (is_left) {
            lx = fminf(lx, sa.x);
            ly = fminf(ly, sa.y);
            lz = fminf(lz, sa.z);
            hx = fmaxf(hx, sb.x);
            hy = fmaxf(hy, sb.y);
            hz = fmaxf(hz, sb.z);
        } else {
            lx = fminf(sa.x, lx);
            ly = fminf(sa.y, ly);
            lz = fminf(sa.z, lz);
            hx = fmaxf(sb.x, hx);
            hy = fmaxf(sb.y, hy);
            hz = fmaxf(sb.z, hz);
        }
        nodes[2 * (size_t)p] = make_float4(lx, ly, lz, __uint_as_float(l));
        nodes[2 * (size_t)p + 1] = make_float4(hx, hy, hz, __uint_as_float(r));
        i = p;
    }
}
#endif

struct BvhWork {
    uint32_t cap = 0;  // prims the arrays hold
    DevMem prims, codes, sorted, order, alt_keys, alt_vals, partial, zeroed, links, parent, nodes, starts, counters,
        scalars, scene;
    uint32_t tiles = 0, nparts = 0;

    int32_t reserve(uint32_t n, int sms);
    // [hist 4*256][tickets 4][pad to 16][look-back 4 * tiles * 256]
    size_t zeroed_bytes() const { return (size_t)(LBVH_PASSES * 256 + 16) * 4 + (size_t)LBVH_PASSES * tiles * 256 * 4; }
    uint32_t* hist() const { return (uint32_t*)zeroed.ptr; }
    uint32_t* tickets() const { return (uint32_t*)zeroed.ptr + LBVH_PASSES * 256; }
    uint32_t* lookback(int pass) const {
        return (uint32_t*)zeroed.ptr + LBVH_PASSES * 256 + 16 + (size_t)pass * tiles * 256;
    }
    uint32_t* depth() const { return (uint32_t*)scalars.ptr; }
    uint32_t* nstarts() const { return (uint32_t*)scalars.ptr + 1; }
};

// The stable radix sort of `codes` over caller-provided work arrays (see
// bvh.cu): order and sorted codes out. Stream-ordered; no allocation.
int32_t enqueue_sort_raw(Ctx* c, const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted,
                         uint32_t* alt_keys, uint32_t* alt_vals, uint32_t* hist, uint32_t* tickets, uint32_t* lookback,
                         uint32_t stride);

// Every stage of Bvh::build over w.prims[0..n) on the context's stream;
// refit = false leaves out the last one, the bounds (the caller runs a
// refit of its own, which must climb as refit_climb does).
int32_t enqueue_build(Ctx* c, BvhWork& w, uint32_t n, uint32_t leaf, Gate gate = Gate{}, bool refit = true);
// Bvh::refit (slots = false: prims through order; true: prims already in
// slot order, Bvh::refit_slots).
int32_t enqueue_refit(Ctx* c, BvhWork& w, uint32_t n, bool slots, Gate gate = Gate{});

}  // namespace phx
