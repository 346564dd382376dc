// The binned SAH builder on the device (phiray src/bvh/sah.rs:25-189,
// Bvh::build_sah): the tree phiray's tracer walks, node for node.
//
// Level by level: every open node of a level is one thread that bins its
// slots, sweeps the 3 x 15 planes, and either becomes a leaf or partitions
// its slots in place (the reference's swap loop) and opens two children in
// the next level's list. Temporary ids come from a counter; once the tree
// is complete, inner-node counts (bottom up) and depth-first ranks (top
// down) give every node the index the reference's work stack hands out,
// and a last bottom-up pass writes the nodes with their bounds.
//
// Nodes under MID slots are one thread each, running the per-node code of
// sah_core.cuh; nodes of MID to BIG slots a block each (64 threads up to
// LARGE slots, 256 above; bins by shared-memory atomics, the swap loop's
// result by the queue model below, in shared memory). Nodes of BIG slots or more —
// the top levels, where a node a thread or warp would leave the GPU idle —
// are cut over blocks of CHUNK slots: the box of centres and the bins are min/max and count reductions
// (exact in any order) merged with atomics; one thread a node then makes
// the reference's decision from those bins (sah_core.cuh decide); and the
// reference's in-place swap partition is reproduced in parallel. That loop
// keeps the left slots in their order, and its right block behaves as a
// queue: from the first right slot on, every slot is an event that appends
// one entry to a log — a right slot appends itself, a left slot moves the
// queue's front entry to the back — so the right block ends as the last
// (count - m) entries of the log, and entry p of a left slot copies entry
// q (its rank among the lefts after the first right). Scans give every
// slot its rank, and pointer jumping over the log's links resolves every
// entry to the slot it carries.
#include <vector>

#include "internal.cuh"
#include "sah_core.cuh"

namespace phx {
namespace {

using sah::TNode;

__global__ void k_sah_init(const float* __restrict__ prims, uint32_t n, float* __restrict__ centres,
                           uint32_t* __restrict__ order) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // Aabb::center (node.rs:90-92)
    for (int k = 0; k < 3; k++) centres[3 * (uint64_t)i + k] = 0.5f * (prims[8 * (uint64_t)i + k] + prims[8 * (uint64_t)i + 4 + k]);
    order[i] = i;
}

__global__ void k_sah_count(const uint32_t* __restrict__ list, uint32_t count, const TNode* __restrict__ tn,
                            uint32_t* inner) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) sah::count_inner(list[k], tn, inner);
}

__global__ void k_sah_place(const uint32_t* __restrict__ list, uint32_t count, const TNode* __restrict__ tn,
                            const uint32_t* __restrict__ inner, uint32_t* rank, uint32_t* final_index) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) sah::place(list[k], tn, inner, rank, final_index);
}

__global__ void k_sah_emit(const uint32_t* __restrict__ list, uint32_t count, const TNode* __restrict__ tn,
                           const uint32_t* __restrict__ final_index, const float* __restrict__ prims,
                           const uint32_t* __restrict__ order, sah::Box* boxes, float* nodes) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) sah::emit(list[k], tn, final_index, prims, order, boxes, nodes);
}

inline uint32_t blocks_of(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

// ---- nodes of BIG slots or more, cut over blocks ----

constexpr uint32_t BIG = 2048;
constexpr uint32_t CHUNK_THREADS = 256;
constexpr uint32_t CHUNK_ITEMS = 8;
constexpr uint32_t CHUNK = CHUNK_THREADS * CHUNK_ITEMS;
constexpr uint32_t HBINS = 3 * sah::BINS;

// A big node of the level and what is decided about it.
struct BigNode {
    uint32_t t, start, end, depth;
    uint32_t cut, axis, at, m, first_right;
    float lo[3], scale[3];
    uint32_t cbox[6];            // box of centres, as ordered words (lo xyz, hi xyz)
    uint32_t bcount[HBINS];      // per axis and bin: slots
    uint32_t bbox[HBINS * 6];    // per axis and bin: the slots' box, as ordered words
};

// A chunk of a big node's slots: [lo, hi) of node b.
struct Chunk {
    uint32_t b, lo, hi;
};

// Floats as words whose unsigned order is the floats' order (for atomic min
// and max; NaN never occurs in a face box).
__device__ __forceinline__ uint32_t ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord(uint32_t w) {
    return __uint_as_float((w & 0x80000000u) ? (w & 0x7FFFFFFFu) : ~w);
}

template <int THREADS = CHUNK_THREADS>
__device__ __forceinline__ uint32_t block_sum_exclusive(uint32_t v, uint32_t* total) {
    __shared__ uint32_t s_warp[THREADS / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? s_warp[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < THREADS / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp ? s_warp[warp - 1] : 0u) + x - v;
    *total = s_warp[THREADS / 32 - 1];
    __syncthreads();
    return before;
}

// ---- nodes of MID to BIG slots: a block a node ----

// Two block forms: 256 threads for nodes of LARGE to BIG slots, 64 threads
// for nodes of MID to LARGE (8 slots a thread either way).
constexpr uint32_t MID = 64;
constexpr uint32_t LARGE = 512;
constexpr uint32_t NODE_ITEMS = 8;  // slots a thread holds
static_assert(256 * NODE_ITEMS == BIG && 64 * NODE_ITEMS == LARGE, "a block holds its largest node");

// sah_core.cuh process for one node by a block: each thread holds 8 of the
// node's slots in registers; the box of centres by block reduction, the bins
// by shared-memory atomics on ordered words (min, max and counts are exact
// in any order), one thread an axis sweeps (sweep_axis) and thread 0 decides
// (decide_from); the reference's swap loop is reproduced in shared memory by
// the queue model (block scan for each slot's rank among the lefts, the
// log's links, pointer jumping in place: a link only ever moves to an
// ancestor on its own chain, so reading a neighbour's already-updated link
// only shortens the chase).
template <int NODE_THREADS>
__global__ void __launch_bounds__(NODE_THREADS, 512 / NODE_THREADS) k_sah_block(
    const uint32_t* __restrict__ list, TNode* tn, const float* __restrict__ prims, const float* __restrict__ centres,
    uint32_t* order, uint32_t leaf, uint32_t* tcount, uint32_t* next, uint32_t* next_count) {
    constexpr uint32_t CAP = NODE_THREADS * NODE_ITEMS;  // slots the block can hold
    __shared__ uint32_t s_count[HBINS];
    __shared__ uint32_t s_box[6 * HBINS];
    __shared__ uint16_t s_ptr[CAP];
    __shared__ uint32_t s_val[CAP];
    __shared__ float s_red[6][NODE_THREADS / 32];
    __shared__ sah::AxisBest s_axis[3];
    __shared__ uint32_t s_cut, s_axis_k, s_at, s_first;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t t = list[blockIdx.x];
    TNode nd = tn[t];
    const uint32_t n = nd.end - nd.start;
    uint32_t m = sah::NONE;
    if (nd.depth + 1 < sah::MAX_DEPTH && n > 1 && n <= CAP) {
        uint32_t slot[NODE_ITEMS];
        const uint32_t j0 = tid * NODE_ITEMS;
        float lo[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
        float hi[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
#pragma unroll
        for (uint32_t e = 0; e < NODE_ITEMS; e++) {
            slot[e] = j0 + e < n ? order[nd.start + j0 + e] : 0u;
            if (j0 + e < n) {
                const float* c = centres + 3 * (uint64_t)slot[e];
                for (int k = 0; k < 3; k++) {
                    lo[k] = fminf(lo[k], c[k]);
                    hi[k] = fmaxf(hi[k], c[k]);
                }
            }
        }
        for (int k = 0; k < 3; k++)
            for (int o = 16; o > 0; o >>= 1) {
                lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            }
        if (lane == 0)
            for (int k = 0; k < 3; k++) {
                s_red[k][warp] = lo[k];
                s_red[3 + k][warp] = hi[k];
            }
        for (uint32_t i = tid; i < HBINS; i += NODE_THREADS) s_count[i] = 0;
        for (uint32_t i = tid; i < 6 * HBINS; i += NODE_THREADS)
            s_box[i] = ord((i % 6) < 3 ? 3.402823466e38f : -3.402823466e38f);
        if (tid == 0) s_first = 0xFFFFFFFFu;
        __syncthreads();
        sah::Box cbox;
        for (int k = 0; k < 3; k++) {
            cbox.lo[k] = s_red[k][0];
            cbox.hi[k] = s_red[3 + k][0];
            for (uint32_t w = 1; w < NODE_THREADS / 32; w++) {
                cbox.lo[k] = fminf(cbox.lo[k], s_red[k][w]);
                cbox.hi[k] = fmaxf(cbox.hi[k], s_red[3 + k][w]);
            }
        }
        float glo[3], scale[3];
        if (!sah::grid_of(cbox, glo, scale)) {
            m = n > leaf ? n / 2 : sah::NONE;
        } else {
#pragma unroll
            for (uint32_t e = 0; e < NODE_ITEMS; e++) {
                if (j0 + e >= n) continue;
                const uint32_t i = slot[e];
                const float* p = prims + 8 * (uint64_t)i;
                for (int k = 0; k < 3; k++) {
                    const uint32_t at = k * sah::BINS + sah::bin_of(centres + 3 * (uint64_t)i, glo, scale, k);
                    atomicAdd(&s_count[at], 1u);
                    for (int f = 0; f < 3; f++) {  // a NaN bound loses, as in f32::min / max
                        if (p[f] == p[f]) atomicMin(&s_box[6 * at + f], ord(p[f]));
                        if (p[4 + f] == p[4 + f]) atomicMax(&s_box[6 * at + 3 + f], ord(p[4 + f]));
                    }
                }
            }
            __syncthreads();
            if (tid < 3) {
                const int k = (int)tid;
                uint32_t mask = 0, bc[sah::BINS];
                sah::Box bb[sah::BINS];
                for (uint32_t a = 0; a < sah::BINS; a++) {
                    const uint32_t i = k * sah::BINS + a;
                    if (!s_count[i]) continue;
                    mask |= 1u << a;
                    bc[a] = s_count[i];
                    for (int f = 0; f < 3; f++) {
                        bb[a].lo[f] = unord(s_box[6 * i + f]);
                        bb[a].hi[f] = unord(s_box[6 * i + 3 + f]);
                    }
                }
                s_axis[k] = scale[k] == 0.0f ? sah::AxisBest{false, 0.0f, 0u} : sah::sweep_axis(mask, bc, bb);
            }
            __syncthreads();
            if (tid == 0) {
                sah::Box bounds = sah::empty_box();
                for (uint32_t a = 0; a < sah::BINS; a++) {
                    if (!s_count[a]) continue;
                    sah::Box b;
                    for (int f = 0; f < 3; f++) {
                        b.lo[f] = unord(s_box[6 * a + f]);
                        b.hi[f] = unord(s_box[6 * a + 3 + f]);
                    }
                    sah::grow(bounds, b);
                }
                const sah::Decision d = sah::decide_from(s_axis, scale, bounds, n, leaf);
                s_cut = d.cut;
                s_axis_k = d.axis;
                s_at = d.at;
            }
            __syncthreads();
            const uint32_t cut = s_cut, axis = s_axis_k, at = s_at;
            if (cut == sah::CUT_HALF) m = n / 2;
            if (cut == sah::CUT_PLANE) {
                bool left[NODE_ITEMS];
                uint32_t mine = 0;
#pragma unroll
                for (uint32_t e = 0; e < NODE_ITEMS; e++) {
                    left[e] = j0 + e < n &&
                              sah::bin_of(centres + 3 * (uint64_t)slot[e], glo, scale, (int)axis) <= at;
                    mine += left[e] ? 1u : 0u;
                    if (j0 + e < n && !left[e]) atomicMin(&s_first, j0 + e);
                }
                uint32_t total = 0;
                uint32_t lr = block_sum_exclusive<NODE_THREADS>(mine, &total);  // (syncs; s_first settles)
                const uint32_t q = total;
                if (q == 0 || q == n) {
                    m = n / 2;  // no left slot or no right one: the swap loop moved nothing
                } else {
                    m = q;
                    const uint32_t first = s_first;
#pragma unroll
                    for (uint32_t e = 0; e < NODE_ITEMS; e++) {
                        const uint32_t j = j0 + e;
                        if (j >= n) continue;
                        if (left[e]) order[nd.start + lr] = slot[e];
                        if (j >= first) {
                            const uint32_t p = j - first;
                            if (left[e]) {
                                s_ptr[p] = (uint16_t)(lr - first);
                            } else {
                                s_ptr[p] = (uint16_t)p;
                                s_val[p] = slot[e];
                            }
                        }
                        if (left[e]) lr++;
                    }
                    __syncthreads();
                    const uint32_t entries = n - first;
                    uint32_t rounds = 1;
                    while ((1u << rounds) < entries) rounds++;
                    for (uint32_t r = 0; r <= rounds; r++) {
                        for (uint32_t x = tid; x < entries; x += NODE_THREADS) s_ptr[x] = s_ptr[s_ptr[x]];
                        __syncthreads();
                    }
                    const uint32_t rotations = m - first;
                    for (uint32_t r = tid; r < n - m; r += NODE_THREADS)
                        order[nd.start + m + r] = s_val[s_ptr[rotations + r]];
                }
            }
        }
    }
    if (tid != 0) return;
    if (m == sah::NONE) {
        nd.left = nd.right = sah::NONE;
    } else {
        const uint32_t c = atomicAdd(tcount, 2u);
        tn[c] = TNode{nd.start, nd.start + m, nd.depth + 1, sah::NONE, sah::NONE};
        tn[c + 1] = TNode{nd.start + m, nd.end, nd.depth + 1, sah::NONE, sah::NONE};
        nd.left = c;
        nd.right = c + 1;
        const uint32_t p = atomicAdd(next_count, 2u);
        next[p] = c;
        next[p + 1] = c + 1;
    }
    tn[t] = nd;
}

// The level's open nodes, split into the big ones (BIG slots or more, not
// at the depth cap) and the rest.
// (counts: small, big, mid, large, and in counts[4] the level's length.)
// The length is `count`, or *dcount when given: the children the level
// before opened, so the host learns them with this level's counts, in one
// wait; the grid then covers an upper bound.
__global__ void k_sah_classify(const uint32_t* __restrict__ list, uint32_t count, const uint32_t* dcount,
                               const TNode* __restrict__ tn, uint32_t* small, uint32_t* big, uint32_t* mid,
                               uint32_t* large, uint32_t* counts) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (dcount) count = *dcount;
    if (k == 0) counts[4] = count;
    if (k >= count) return;
    const uint32_t t = list[k];
    const TNode nd = tn[t];
    const uint32_t n = nd.end - nd.start;
    const bool open = nd.depth + 1 < sah::MAX_DEPTH;
    if (open && n >= BIG) big[atomicAdd(counts + 1, 1u)] = t;
    else if (open && n >= LARGE) large[atomicAdd(counts + 3, 1u)] = t;
    else if (open && n >= MID) mid[atomicAdd(counts + 2, 1u)] = t;
    else small[atomicAdd(counts, 1u)] = t;
}

// Nodes under MID slots (and nodes at the depth cap): a thread a node,
// sah_core.cuh process as it is.
struct DeviceAdd {
    __device__ uint32_t operator()(uint32_t* p, uint32_t v) const { return atomicAdd(p, v); }
};

__global__ void k_sah_thread(const uint32_t* __restrict__ list, uint32_t count, TNode* tn,
                             const float* __restrict__ prims, const float* __restrict__ centres, uint32_t* order,
                             uint32_t leaf, uint32_t* tcount, uint32_t* next, uint32_t* next_count) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    sah::process(list[k], tn, prims, centres, order, leaf, tcount, next, next_count, DeviceAdd{});
}

__global__ void k_big_setup(const uint32_t* __restrict__ big, uint32_t nb, const TNode* __restrict__ tn,
                            BigNode* bn, uint2* spans) {
    const uint32_t b = blockIdx.x;
    if (b >= nb) return;
    BigNode& B = bn[b];
    if (threadIdx.x == 0) {
        const TNode nd = tn[big[b]];
        spans[b] = make_uint2(nd.start, nd.end);
        B.t = big[b];
        B.start = nd.start;
        B.end = nd.end;
        B.depth = nd.depth;
        B.cut = sah::CUT_LEAF;
        B.axis = B.at = B.m = 0;
        B.first_right = 0xFFFFFFFFu;
        for (int k = 0; k < 3; k++) {
            B.cbox[k] = ord(3.402823466e38f);
            B.cbox[3 + k] = ord(-3.402823466e38f);
        }
    }
    for (uint32_t i = threadIdx.x; i < HBINS; i += blockDim.x) B.bcount[i] = 0;
    for (uint32_t i = threadIdx.x; i < HBINS * 6; i += blockDim.x)
        B.bbox[i] = ord((i % 6) < 3 ? 3.402823466e38f : -3.402823466e38f);
}

// Box of a big node's centres (sah.rs:121-123).
__global__ void __launch_bounds__(CHUNK_THREADS) k_big_cbox(const Chunk* __restrict__ chunks, BigNode* bn,
                                                            const float* __restrict__ centres,
                                                            const uint32_t* __restrict__ order) {
    const Chunk ch = chunks[blockIdx.x];
    float lo[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
    float hi[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    for (uint32_t j = ch.lo + threadIdx.x; j < ch.hi; j += CHUNK_THREADS) {
        const float* c = centres + 3 * (uint64_t)order[j];
        for (int k = 0; k < 3; k++) {
            lo[k] = fminf(lo[k], c[k]);
            hi[k] = fmaxf(hi[k], c[k]);
        }
    }
    for (int k = 0; k < 3; k++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    if ((threadIdx.x & 31u) == 0) {
        BigNode& B = bn[ch.b];
        for (int k = 0; k < 3; k++) {
            atomicMin(&B.cbox[k], ord(lo[k]));
            atomicMax(&B.cbox[3 + k], ord(hi[k]));
        }
    }
}

// Grid::of per big node; a flat node (one point) is halved or a leaf.
__global__ void k_big_grid(BigNode* bn, uint32_t nb, uint32_t leaf) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    BigNode& B = bn[b];
    sah::Box cb;
    for (int k = 0; k < 3; k++) {
        cb.lo[k] = unord(B.cbox[k]);
        cb.hi[k] = unord(B.cbox[3 + k]);
    }
    const uint32_t count = B.end - B.start;
    if (!sah::grid_of(cb, B.lo, B.scale)) {
        B.cut = count > leaf ? sah::CUT_HALF : sah::CUT_LEAF;
        B.m = count / 2;
        B.first_right = 0xFFFFFFFEu;  // decided: no bins
    }
}

// The bins of a big node (sah.rs:128-140): per axis and bin, the slots and
// the union of their boxes.
__global__ void __launch_bounds__(CHUNK_THREADS) k_big_bins(const Chunk* __restrict__ chunks, BigNode* bn,
                                                            const float* __restrict__ prims,
                                                            const float* __restrict__ centres,
                                                            const uint32_t* __restrict__ order) {
    __shared__ uint32_t s_count[HBINS];
    __shared__ uint32_t s_box[HBINS * 6];
    const Chunk ch = chunks[blockIdx.x];
    BigNode& B = bn[ch.b];
    if (B.first_right == 0xFFFFFFFEu) return;  // decided on its grid
    for (uint32_t i = threadIdx.x; i < HBINS; i += CHUNK_THREADS) s_count[i] = 0;
    for (uint32_t i = threadIdx.x; i < HBINS * 6; i += CHUNK_THREADS)
        s_box[i] = ord((i % 6) < 3 ? 3.402823466e38f : -3.402823466e38f);
    __syncthreads();
    const float lo[3] = {B.lo[0], B.lo[1], B.lo[2]}, scale[3] = {B.scale[0], B.scale[1], B.scale[2]};
    for (uint32_t j = ch.lo + threadIdx.x; j < ch.hi; j += CHUNK_THREADS) {
        const uint32_t i = order[j];
        const float* p = prims + 8 * (uint64_t)i;
        for (int k = 0; k < 3; k++) {
            const uint32_t at = k * sah::BINS + sah::bin_of(centres + 3 * (uint64_t)i, lo, scale, k);
            atomicAdd(&s_count[at], 1u);
            for (int e = 0; e < 3; e++) {  // a NaN bound loses, as in f32::min / max
                if (p[e] == p[e]) atomicMin(&s_box[6 * at + e], ord(p[e]));
                if (p[4 + e] == p[4 + e]) atomicMax(&s_box[6 * at + 3 + e], ord(p[4 + e]));
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < HBINS; i += CHUNK_THREADS)
        if (s_count[i]) atomicAdd(&B.bcount[i], s_count[i]);
    for (uint32_t i = threadIdx.x; i < HBINS * 6; i += CHUNK_THREADS) {
        if (!s_count[i / 6]) continue;
        if ((i % 6) < 3) atomicMin(&B.bbox[i], s_box[i]);
        else atomicMax(&B.bbox[i], s_box[i]);
    }
}

// One thread a big node: the reference's decision from the bins, the left
// count, and the children's entries (as sah_core.cuh process makes them).
__global__ void k_big_choose(BigNode* bn, uint32_t nb, TNode* tn, uint32_t leaf, uint32_t* tcount, uint32_t* next,
                             uint32_t* next_count) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    BigNode& B = bn[b];
    const uint32_t count = B.end - B.start;
    if (B.first_right != 0xFFFFFFFEu) {
        uint32_t bcount[3][sah::BINS];
        sah::Box bbox[3][sah::BINS];
        for (int k = 0; k < 3; k++)
            for (uint32_t a = 0; a < sah::BINS; a++) {
                const uint32_t i = k * sah::BINS + a;
                bcount[k][a] = B.bcount[i];
                for (int e = 0; e < 3; e++) {
                    bbox[k][a].lo[e] = unord(B.bbox[6 * i + e]);
                    bbox[k][a].hi[e] = unord(B.bbox[6 * i + 3 + e]);
                }
            }
        const sah::Decision d = sah::decide(bcount, bbox, B.scale, count, leaf);
        B.cut = d.cut;
        B.axis = d.axis;
        B.at = d.at;
        if (d.cut == sah::CUT_HALF) B.m = count / 2;
        if (d.cut == sah::CUT_PLANE) {
            uint32_t m = 0;
            for (uint32_t a = 0; a <= d.at; a++) m += bcount[d.axis][a];
            // no left slot or no right one: the swap loop moved nothing
            if (m == 0 || m == count) {
                B.cut = sah::CUT_HALF;
                m = count / 2;
            }
            B.m = m;
        }
    }
    TNode nd = tn[B.t];
    if (B.cut == sah::CUT_LEAF) {
        nd.left = nd.right = sah::NONE;
    } else {
        const uint32_t c = atomicAdd(tcount, 2u);
        tn[c] = TNode{nd.start, nd.start + B.m, nd.depth + 1, sah::NONE, sah::NONE};
        tn[c + 1] = TNode{nd.start + B.m, nd.end, nd.depth + 1, sah::NONE, sah::NONE};
        nd.left = c;
        nd.right = c + 1;
        const uint32_t p = atomicAdd(next_count, 2u);
        next[p] = c;
        next[p + 1] = c + 1;
    }
    tn[B.t] = nd;
}

__device__ __forceinline__ bool goes_left(const BigNode& B, const float* centres, uint32_t slot_prim) {
    return sah::bin_of(centres + 3 * (uint64_t)slot_prim, B.lo, B.scale, (int)B.axis) <= B.at;
}

// Partition, step 1: each chunk's left slots ranked in the chunk, the
// chunk's count of them, and the node's first right slot.
__global__ void __launch_bounds__(CHUNK_THREADS) k_part_flags(const Chunk* __restrict__ chunks, BigNode* bn,
                                                              const float* __restrict__ centres,
                                                              const uint32_t* __restrict__ order,
                                                              uint32_t* __restrict__ rank, uint32_t* chunk_lefts) {
    const Chunk ch = chunks[blockIdx.x];
    BigNode& B = bn[ch.b];
    if (B.cut != sah::CUT_PLANE) return;
    const uint32_t j0 = ch.lo + threadIdx.x * CHUNK_ITEMS;
    uint32_t mine = 0, first = 0xFFFFFFFFu;
    bool left[CHUNK_ITEMS];
#pragma unroll
    for (uint32_t e = 0; e < CHUNK_ITEMS; e++) {
        const uint32_t j = j0 + e;
        left[e] = j < ch.hi && goes_left(B, centres, order[j]);
        if (j < ch.hi && !left[e] && first == 0xFFFFFFFFu) first = j;
        mine += left[e] ? 1u : 0u;
    }
    uint32_t total = 0;
    uint32_t before = block_sum_exclusive(mine, &total);
#pragma unroll
    for (uint32_t e = 0; e < CHUNK_ITEMS; e++) {
        const uint32_t j = j0 + e;
        if (j < ch.hi) rank[j] = before;
        if (left[e]) before++;
    }
    if (threadIdx.x == 0) chunk_lefts[blockIdx.x] = total;
    for (int o = 16; o > 0; o >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
    if ((threadIdx.x & 31u) == 0 && first != 0xFFFFFFFFu) atomicMin(&B.first_right, first);
}

// Partition, step 2 (a thread a chunk): the chunk's left count before it
// within its node (the table lists a node's chunks in order, so they are the
// chunks before it with the same node).
__global__ void k_part_chunks(const Chunk* __restrict__ chunks, uint32_t nchunks, const uint32_t* __restrict__ lefts,
                              uint32_t* offs) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const uint32_t node = chunks[c].b;
    uint32_t run = 0;
    for (uint32_t k = c; k-- > 0 && chunks[k].b == node;) run += lefts[k];
    offs[c] = run;
}

// Partition, step 3: left slots to their places; from the first right slot
// on, every slot's log entry (a right slot carries itself; a left slot
// links to the entry its rotation copies).
__global__ void __launch_bounds__(CHUNK_THREADS) k_part_scatter(const Chunk* __restrict__ chunks,
                                                                const BigNode* __restrict__ bn,
                                                                const float* __restrict__ centres,
                                                                const uint32_t* __restrict__ order,
                                                                const uint32_t* __restrict__ rank,
                                                                const uint32_t* __restrict__ offs, uint32_t* out,
                                                                uint32_t* ptr, uint32_t* val) {
    const Chunk ch = chunks[blockIdx.x];
    const BigNode& B = bn[ch.b];
    if (B.cut != sah::CUT_PLANE) return;
    const uint32_t first = B.first_right - B.start;  // lefts before the first right
    for (uint32_t j = ch.lo + threadIdx.x; j < ch.hi; j += CHUNK_THREADS) {
        const uint32_t slot = order[j];
        const bool left = goes_left(B, centres, slot);
        const uint32_t lr = offs[blockIdx.x] + rank[j];  // lefts before j in the node
        if (left) out[B.start + lr] = slot;
        const uint32_t jr = j - B.start;
        if (jr >= first) {
            const uint32_t p = B.start + (jr - first);
            if (left) {
                ptr[p] = B.start + (lr - first);
            } else {
                ptr[p] = p;
                val[p] = slot;
            }
        }
    }
}

// Partition, step 4: one round of pointer jumping over the log's links.
__global__ void __launch_bounds__(CHUNK_THREADS) k_part_jump(const Chunk* __restrict__ chunks,
                                                             const BigNode* __restrict__ bn,
                                                             const uint32_t* __restrict__ src, uint32_t* dst) {
    const Chunk ch = chunks[blockIdx.x];
    const BigNode& B = bn[ch.b];
    if (B.cut != sah::CUT_PLANE) return;
    const uint32_t end = B.start + (B.end - B.first_right);  // the log's entries
    for (uint32_t x = ch.lo + threadIdx.x; x < ch.hi && x < end; x += CHUNK_THREADS) dst[x] = src[src[x]];
}

// Partition, step 5: the right block is the log's last (count - m) entries.
__global__ void __launch_bounds__(CHUNK_THREADS) k_part_rights(const Chunk* __restrict__ chunks,
                                                               const BigNode* __restrict__ bn,
                                                               const uint32_t* __restrict__ ptr,
                                                               const uint32_t* __restrict__ val, uint32_t* out) {
    const Chunk ch = chunks[blockIdx.x];
    const BigNode& B = bn[ch.b];
    if (B.cut != sah::CUT_PLANE) return;
    const uint32_t first = B.first_right - B.start;
    const uint32_t rotations = B.m - first;
    for (uint32_t x = ch.lo + threadIdx.x; x < ch.hi; x += CHUNK_THREADS) {
        if (x < B.start + B.m) continue;
        const uint32_t r = x - (B.start + B.m);
        out[x] = val[ptr[B.start + rotations + r]];
    }
}

__global__ void __launch_bounds__(CHUNK_THREADS) k_part_copy(const Chunk* __restrict__ chunks,
                                                             const BigNode* __restrict__ bn,
                                                             const uint32_t* __restrict__ src, uint32_t* order) {
    const Chunk ch = chunks[blockIdx.x];
    if (bn[ch.b].cut != sah::CUT_PLANE) return;
    for (uint32_t x = ch.lo + threadIdx.x; x < ch.hi; x += CHUNK_THREADS) order[x] = src[x];
}

}  // namespace
}  // namespace phx

using namespace phx;

extern "C" {

int32_t phx_bvh_build_sah(phx_ctx ctx, const phx_aabb* prims, uint32_t n, uint32_t leaf, phx_node* nodes,
                          uint32_t* order, uint32_t* node_count, uint32_t* depth) {
    if (!ctx || !node_count || !depth || (n && (!prims || !nodes || !order)))
        return fail(PHX_ERR_INVALID, "null argument");
    if (n >= (1u << 30)) return fail(PHX_ERR_INVALID, "too many primitives");
    *node_count = 0;
    *depth = 0;
    if (n == 0) return PHX_OK;
    PHX_TRY(use(&ctx->c));
    Ctx* c = &ctx->c;
    cudaStream_t s = c->stream;
    const uint32_t cap = 2 * n - 1;
    DevMem centres, tn, lists, counters, inner, rank, final_index, boxes;
    PHX_TRY(centres.reserve((size_t)n * 12));
    PHX_TRY(tn.reserve((size_t)cap * sizeof(TNode)));
    PHX_TRY(lists.reserve((size_t)cap * 4));
    PHX_TRY(counters.reserve(8));
    PHX_TRY(inner.reserve((size_t)cap * 4));
    PHX_TRY(rank.reserve((size_t)cap * 4));
    PHX_TRY(final_index.reserve((size_t)cap * 4));
    PHX_TRY(boxes.reserve((size_t)cap * sizeof(sah::Box)));
    const float* P = (const float*)prims;
    TNode* T = (TNode*)tn.ptr;
    uint32_t* L = (uint32_t*)lists.ptr;
    uint32_t* cnt = (uint32_t*)counters.ptr;  // [0] temporary ids handed out, [1] next level's length
    k_sah_init<<<blocks_of(n, 256), 256, 0, s>>>(P, n, (float*)centres.ptr, order);
    const TNode root{0, n, 0, sah::NONE, sah::NONE};
    const uint32_t zero = 0, one = 1;
    PHX_CUDA(cudaMemcpyAsync(T, &root, sizeof root, cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(L, &zero, 4, cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(cnt, &one, 4, cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(rank.ptr, &zero, 4, cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(final_index.ptr, &zero, 4, cudaMemcpyHostToDevice, s));
    // Levels: list offsets and lengths (at most MAX_DEPTH levels: a node at
    // depth 31 is a leaf).
    // Big-node work arrays (sized for the widest level: at most n / BIG big
    // nodes, n / CHUNK + n / BIG chunks).
    const uint32_t max_big = n / BIG + 1, max_chunks = n / CHUNK + max_big + 1;
    DevMem small_list, mid_list, large_list, big_list, lcounts, bnodes, spans, chunks, rank_w, lefts, offs, out_w,
        ptr_a, ptr_b, val_w;
    PHX_TRY(small_list.reserve((size_t)cap * 4));
    PHX_TRY(mid_list.reserve((size_t)(n / MID + 1) * 4));
    PHX_TRY(large_list.reserve((size_t)(n / LARGE + 1) * 4));
    PHX_TRY(lcounts.reserve(20));
    if (n >= BIG) {
        PHX_TRY(spans.reserve((size_t)max_big * 8));
        PHX_TRY(big_list.reserve((size_t)max_big * 4));
        PHX_TRY(bnodes.reserve((size_t)max_big * sizeof(BigNode)));
        PHX_TRY(chunks.reserve((size_t)max_chunks * sizeof(Chunk)));
        PHX_TRY(rank_w.reserve((size_t)n * 4));
        PHX_TRY(lefts.reserve((size_t)max_chunks * 4));
        PHX_TRY(offs.reserve((size_t)max_chunks * 4));
        PHX_TRY(out_w.reserve((size_t)n * 4));
        PHX_TRY(ptr_a.reserve((size_t)n * 4));
        PHX_TRY(ptr_b.reserve((size_t)n * 4));
        PHX_TRY(val_w.reserve((size_t)n * 4));
    }
    std::vector<uint32_t> off{0}, len{1};
    std::vector<uint2> host_big;
    std::vector<Chunk> host_chunks;
    // Level 0's classification; each level then classifies the next one
    // right behind its own kernels, and one wait a level reads both the
    // children opened and their classes.
    PHX_CUDA(cudaMemsetAsync(lcounts.ptr, 0, 16, s));
    k_sah_classify<<<1, 256, 0, s>>>(L, 1u, nullptr, T, (uint32_t*)small_list.ptr, (uint32_t*)big_list.ptr,
                                     (uint32_t*)mid_list.ptr, (uint32_t*)large_list.ptr, (uint32_t*)lcounts.ptr);
    for (uint32_t lv = 0; lv < sah::MAX_DEPTH; lv++) {
        uint32_t lc[5] = {0, 0, 0, 0, 0};
        PHX_CUDA(cudaMemcpyAsync(lc, lcounts.ptr, 20, cudaMemcpyDeviceToHost, s));
        PHX_TRY(wait_stream(s, 0));
        if (lv > 0) {
            // lc[4]: the children the level before opened (this level's length)
            if (lc[4] == 0) break;
            const uint32_t at = off[lv - 1] + len[lv - 1];
            if (at + lc[4] > cap) return fail(PHX_ERR_DEVICE, "SAH build: more nodes than 2n - 1");
            off.push_back(at);
            len.push_back(lc[4]);
        }
        const uint32_t next = off[lv] + len[lv];
        PHX_CUDA(cudaMemsetAsync(cnt + 1, 0, 4, s));
        const uint32_t* level = (const uint32_t*)small_list.ptr;
        uint32_t nsmall = 0, nmid = 0, nlarge = 0;
        {
            nsmall = lc[0];
            nmid = lc[2];
            nlarge = lc[3];
            const uint32_t nb = lc[1];
            if (nb) {
                BigNode* BN = (BigNode*)bnodes.ptr;
                k_big_setup<<<nb, 256, 0, s>>>((const uint32_t*)big_list.ptr, nb, T, BN, (uint2*)spans.ptr);
                host_big.resize(nb);
                PHX_CUDA(cudaMemcpyAsync(host_big.data(), spans.ptr, (size_t)nb * 8, cudaMemcpyDeviceToHost, s));
                PHX_TRY(wait_stream(s, 0));
                host_chunks.clear();
                uint32_t widest = 0;
                for (uint32_t b = 0; b < nb; b++) {
                    const uint32_t lo = host_big[b].x, hi = host_big[b].y;
                    widest = std::max(widest, hi - lo);
                    for (uint32_t j = lo; j < hi; j += CHUNK) host_chunks.push_back(Chunk{b, j, std::min(j + CHUNK, hi)});
                }
                const uint32_t nc = (uint32_t)host_chunks.size();
                if (nc > max_chunks) return fail(PHX_ERR_DEVICE, "SAH build: chunk table overflow");
                Chunk* CH = (Chunk*)chunks.ptr;
                PHX_CUDA(cudaMemcpyAsync(CH, host_chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice, s));
                const float* Cc = (const float*)centres.ptr;
                k_big_cbox<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, Cc, order);
                k_big_grid<<<blocks_of(nb, 64), 64, 0, s>>>(BN, nb, leaf);
                k_big_bins<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, P, Cc, order);
                k_big_choose<<<blocks_of(nb, 64), 64, 0, s>>>(BN, nb, T, leaf, cnt, L + next, cnt + 1);
                uint32_t* R = (uint32_t*)rank_w.ptr;
                k_part_flags<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, Cc, order, R, (uint32_t*)lefts.ptr);
                k_part_chunks<<<blocks_of(nc, 128), 128, 0, s>>>(CH, nc, (const uint32_t*)lefts.ptr,
                                                                 (uint32_t*)offs.ptr);
                uint32_t* pa = (uint32_t*)ptr_a.ptr;
                uint32_t* pb = (uint32_t*)ptr_b.ptr;
                k_part_scatter<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, Cc, order, R, (const uint32_t*)offs.ptr,
                                                            (uint32_t*)out_w.ptr, pa, (uint32_t*)val_w.ptr);
                uint32_t rounds = 1;
                while ((1u << rounds) < widest) rounds++;
                for (uint32_t r = 0; r <= rounds; r++) {
                    k_part_jump<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, pa, pb);
                    std::swap(pa, pb);
                }
                k_part_rights<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, pa, (const uint32_t*)val_w.ptr,
                                                           (uint32_t*)out_w.ptr);
                k_part_copy<<<nc, CHUNK_THREADS, 0, s>>>(CH, BN, (const uint32_t*)out_w.ptr, order);
                PHX_CUDA(cudaGetLastError());
            }
        }
        if (nlarge)
            k_sah_block<256><<<nlarge, 256, 0, s>>>((const uint32_t*)large_list.ptr, T, P, (const float*)centres.ptr,
                                                    order, leaf, cnt, L + next, cnt + 1);
        if (nmid)
            k_sah_block<64><<<nmid, 64, 0, s>>>((const uint32_t*)mid_list.ptr, T, P, (const float*)centres.ptr, order,
                                                leaf, cnt, L + next, cnt + 1);
        if (nsmall)
            k_sah_thread<<<blocks_of(nsmall, 64), 64, 0, s>>>(level, nsmall, T, P, (const float*)centres.ptr, order,
                                                              leaf, cnt, L + next, cnt + 1);
        PHX_CUDA(cudaGetLastError());
        // the next level: its length is the children just opened (cnt[1]);
        // at most two a node of this level
        PHX_CUDA(cudaMemsetAsync(lcounts.ptr, 0, 16, s));
        k_sah_classify<<<blocks_of(2 * len[lv], 256), 256, 0, s>>>(
            L + next, 0u, cnt + 1, T, (uint32_t*)small_list.ptr, (uint32_t*)big_list.ptr, (uint32_t*)mid_list.ptr,
            (uint32_t*)large_list.ptr, (uint32_t*)lcounts.ptr);
        PHX_CUDA(cudaGetLastError());
    }
    const uint32_t levels = (uint32_t)len.size();
    for (uint32_t lv = levels; lv-- > 0;)
        k_sah_count<<<blocks_of(len[lv], 256), 256, 0, s>>>(L + off[lv], len[lv], T, (uint32_t*)inner.ptr);
    for (uint32_t lv = 0; lv < levels; lv++)
        k_sah_place<<<blocks_of(len[lv], 256), 256, 0, s>>>(L + off[lv], len[lv], T, (const uint32_t*)inner.ptr,
                                                            (uint32_t*)rank.ptr, (uint32_t*)final_index.ptr);
    for (uint32_t lv = levels; lv-- > 0;)
        k_sah_emit<<<blocks_of(len[lv], 256), 256, 0, s>>>(L + off[lv], len[lv], T, (const uint32_t*)final_index.ptr, P,
                                                           order, (sah::Box*)boxes.ptr, (float*)nodes);
    PHX_CUDA(cudaGetLastError());
    uint32_t total = 0;
    PHX_CUDA(cudaMemcpyAsync(&total, cnt, 4, cudaMemcpyDeviceToHost, s));
    PHX_TRY(wait_stream(s, 0));
    *node_count = total;
    *depth = levels - 1;
    return read_status(c);
}

}  // extern "C"
