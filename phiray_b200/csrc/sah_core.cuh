// The binned SAH builder's per-node steps (phiray src/bvh/sah.rs:25-189),
// written once for the device kernels of sah.cu and for a host build of
// the same code: every function here is plain arithmetic on one node or
// one tree entry, so a host loop over the entries computes exactly what a
// launch over them computes.
//
// The tree equals the reference's node for node: the same bins, sweep and
// leaf rule per node, the same in-place (swap) partition of the node's
// slots, and node indices in the order the reference's work stack hands
// them out (children of the k-th inner node in depth-first, left-first
// order at 2k + 1 and 2k + 2).
#pragma once

#include <stdint.h>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

#define SAH_HD __host__ __device__ __forceinline__

namespace phx {
namespace sah {

constexpr uint32_t BINS = 16;        // sah.rs:26 BIN_COUNT
constexpr float TRAVERSE = 1.0f;     // sah.rs:30
constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t LEAF_BIT = 0x80000000u;
constexpr uint32_t MAX_DEPTH = 32;   // node.rs STACK: a node at depth 31 is a leaf

// Rust f32::min / max: the argument that is not NaN wins.
SAH_HD float rmin(float a, float b) { return a != a ? b : (b != b ? a : (a < b ? a : b)); }
SAH_HD float rmax(float a, float b) { return a != a ? b : (b != b ? a : (a > b ? a : b)); }

struct Box {
    float lo[3], hi[3];
};

SAH_HD Box empty_box() {
    Box b;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = 3.402823466e38f;    // f32::MAX
        b.hi[k] = -3.402823466e38f;   // f32::MIN
    }
    return b;
}

SAH_HD void grow(Box& b, const Box& o) {
    for (int k = 0; k < 3; k++) {
        b.lo[k] = rmin(b.lo[k], o.lo[k]);
        b.hi[k] = rmax(b.hi[k], o.hi[k]);
    }
}

// A primitive's box from phiray's Aabb layout: lo.xyz, pad, hi.xyz, pad.
SAH_HD Box prim_box(const float* aabb8) {
    Box b;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = aabb8[k];
        b.hi[k] = aabb8[4 + k];
    }
    return b;
}

// sah.rs:32-35
SAH_HD float area(const Box& b) {
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = rmax(b.hi[k] - b.lo[k], 0.0f);
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
}

// sah.rs:68-79: the bin of centre c along axis k (Rust `as usize`
// truncates toward zero and saturates; NaN gives 0).
SAH_HD uint32_t bin_of(const float* c, const float* lo, const float* scale, int k) {
    const float v = (c[k] - lo[k]) * scale[k];
    const uint32_t b = (v != v || v <= 0.0f) ? 0u : (v >= 16.0f ? BINS - 1 : (uint32_t)v);
    return b < BINS - 1 ? b : BINS - 1;
}

// Grid::of (sah.rs:40-66): the bins' origin and scale from a node's box of
// centres; true when every centre sits in one point (no plane separates).
SAH_HD bool grid_of(const Box& cbox, float* lo, float* scale) {
    bool flat = true;
    for (int k = 0; k < 3; k++) {
        const float e = cbox.hi[k] - cbox.lo[k];
        lo[k] = cbox.lo[k];
        scale[k] = e > 0.0f ? (float)BINS * (1.0f - 1e-5f) / e : 0.0f;
        if (scale[k] != 0.0f) flat = false;
    }
    return !flat;
}

// What split does with a node once its bins are filled (sah.rs:150-181):
// the cheapest plane over the three axes' sweeps, then the leaf rule.
enum Cut : uint32_t { CUT_LEAF = 0, CUT_HALF = 1, CUT_PLANE = 2 };
struct Decision {
    uint32_t cut, axis, at;
};

SAH_HD Decision decide(const uint32_t (*bcount)[BINS], const Box (*bbox)[BINS], const float* scale, uint32_t count,
                       uint32_t leaf) {
    bool have = false;
    float best = 0.0f;
    uint32_t best_k = 0;
    uint32_t best_at = 0;
    for (int k = 0; k < 3; k++) {
        if (scale[k] == 0.0f) continue;
        float right_area[BINS];
        uint32_t right_count[BINS];
        Box b = empty_box();
        uint32_t c = 0;
        for (uint32_t at = BINS - 1; at >= 1; at--) {
            grow(b, bbox[k][at]);
            c += bcount[k][at];
            right_area[at] = area(b);
            right_count[at] = c;
        }
        b = empty_box();
        c = 0;
        for (uint32_t at = 0; at + 1 < BINS; at++) {
            grow(b, bbox[k][at]);
            c += bcount[k][at];
            const uint32_t rc = right_count[at + 1];
            if (c == 0 || rc == 0) continue;
            const float cost = area(b) * (float)c + right_area[at + 1] * (float)rc;
            if (!have || cost < best) {
                have = true;
                best = cost;
                best_k = (uint32_t)k;
                best_at = at;
            }
        }
    }
    Box bounds = empty_box();
    for (uint32_t b = 0; b < BINS; b++) grow(bounds, bbox[0][b]);
    if (!have) return Decision{count > leaf ? (uint32_t)CUT_HALF : (uint32_t)CUT_LEAF, 0u, 0u};
    const float parent = rmax(area(bounds), 1.17549435e-38f);  // f32::MIN_POSITIVE
    if (count <= leaf && TRAVERSE + best / parent >= (float)count) return Decision{CUT_LEAF, 0u, 0u};
    return Decision{CUT_PLANE, best_k, best_at};
}

SAH_HD uint32_t lowest_bit(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)(__ffs((int)x) - 1);
#else
    return (uint32_t)__builtin_ctz(x);
#endif
}

// One axis of the sweep (sah.rs:150-170) over the occupied bins only
// (mask bit b: bin b holds a slot; the entries of empty bins are never
// read): the first plane of least cost in ascending order. An empty bin adds
// nothing to a union or a count, so every plane between two occupied bins
// prices as the plane at the lower one, which the ascending strict-`<` sweep
// meets first; planes below the first occupied bin or at and above the last
// have an empty side and are skipped.
struct AxisBest {
    bool have;
    float cost;
    uint32_t at;
};

SAH_HD AxisBest sweep_axis(uint32_t mask, const uint32_t* bcount, const Box* bbox) {
    AxisBest r{false, 0.0f, 0u};
    float right_area[BINS];
    uint32_t right_count[BINS];
    Box b = empty_box();
    uint32_t c = 0;
    for (uint32_t at = BINS; at-- > 0;) {
        if (!((mask >> at) & 1u)) continue;
        grow(b, bbox[at]);
        c += bcount[at];
        right_area[at] = area(b);
        right_count[at] = c;
    }
    b = empty_box();
    c = 0;
    for (uint32_t at = 0; at + 1 < BINS; at++) {
        if (!((mask >> at) & 1u)) continue;
        grow(b, bbox[at]);
        c += bcount[at];
        const uint32_t above = mask & ~((2u << at) - 1u);  // occupied bins past `at`
        if (!above) break;
        const uint32_t nxt = lowest_bit(above);
        const float cost = area(b) * (float)c + right_area[nxt] * (float)right_count[nxt];
        if (!r.have || cost < r.cost) r = AxisBest{true, cost, at};
    }
    return r;
}

// The decision from the three axes' sweeps (axis k skipped where scale[k]
// is 0): the reference keeps the first plane of least cost over the axes in
// order (strict `<`), i.e. the axis with the least cost, the lower axis on a
// tie; then the leaf rule against the node's bounds.
SAH_HD Decision decide_from(const AxisBest* axes, const float* scale, const Box& bounds, uint32_t count,
                            uint32_t leaf) {
    bool have = false;
    float best = 0.0f;
    uint32_t best_k = 0, best_at = 0;
    for (int k = 0; k < 3; k++) {
        if (scale[k] == 0.0f || !axes[k].have) continue;
        if (!have || axes[k].cost < best) {
            have = true;
            best = axes[k].cost;
            best_k = (uint32_t)k;
            best_at = axes[k].at;
        }
    }
    if (!have) return Decision{count > leaf ? (uint32_t)CUT_HALF : (uint32_t)CUT_LEAF, 0u, 0u};
    const float parent = rmax(area(bounds), 1.17549435e-38f);  // f32::MIN_POSITIVE
    if (count <= leaf && TRAVERSE + best / parent >= (float)count) return Decision{CUT_LEAF, 0u, 0u};
    return Decision{CUT_PLANE, best_k, best_at};
}

// decide over the occupied bins only (mask[k] for axis k).
SAH_HD Decision decide_occupied(const uint32_t* mask, const uint32_t (*bcount)[BINS], const Box (*bbox)[BINS],
                                const float* scale, uint32_t count, uint32_t leaf) {
    AxisBest axes[3];
    for (int k = 0; k < 3; k++)
        axes[k] = scale[k] == 0.0f ? AxisBest{false, 0.0f, 0u} : sweep_axis(mask[k], bcount[k], bbox[k]);
    Box bounds = empty_box();
    for (uint32_t b = 0; b < BINS; b++)
        if ((mask[0] >> b) & 1u) grow(bounds, bbox[0][b]);
    return decide_from(axes, scale, bounds, count, leaf);
}

// sah.rs:114-189 split: the left count after reordering slots[0, count), or
// NONE for a leaf. Serial over the node's slots; a bin's entries are set
// when the first slot lands in it (so a small node touches only its
// occupied bins).
SAH_HD uint32_t split(const float* prims, const float* centres, uint32_t* slots, uint32_t count, uint32_t leaf) {
    if (count <= 1) return NONE;
    Box cbox = empty_box();
#pragma unroll 4
    for (uint32_t j = 0; j < count; j++) {
        const float* c = centres + 3 * (uint64_t)slots[j];
        Box p;
        for (int k = 0; k < 3; k++) p.lo[k] = p.hi[k] = c[k];
        grow(cbox, p);
    }
    float lo[3], scale[3];
    if (!grid_of(cbox, lo, scale)) return count > leaf ? count / 2 : NONE;
    // One axis at a time (its 16 bins, then its sweep), so a thread keeps a
    // third of the bins live; the bins of an axis and the decision are those
    // of all three filled together.
    AxisBest axes[3];
    Box bounds = empty_box();
    for (int k = 0; k < 3; k++) {
        axes[k] = AxisBest{false, 0.0f, 0u};
        if (scale[k] == 0.0f && k != 0) continue;  // (axis 0's bins give the node's bounds)
        uint32_t mask = 0u;
        uint32_t bcount[BINS];
        Box bbox[BINS];
#pragma unroll 4
        for (uint32_t j = 0; j < count; j++) {
            const uint32_t i = slots[j];
            const uint32_t at = bin_of(centres + 3 * (uint64_t)i, lo, scale, k);
            const Box pb = prim_box(prims + 8 * (uint64_t)i);
            if (!((mask >> at) & 1u)) {
                mask |= 1u << at;
                bcount[at] = 0;
                bbox[at] = empty_box();
            }
            bcount[at] += 1;
            grow(bbox[at], pb);
        }
        if (k == 0)
            for (uint32_t b = 0; b < BINS; b++)
                if ((mask >> b) & 1u) grow(bounds, bbox[b]);
        if (scale[k] != 0.0f) axes[k] = sweep_axis(mask, bcount, bbox);
    }
    const Decision d = decide_from(axes, scale, bounds, count, leaf);
    if (d.cut == CUT_LEAF) return NONE;
    if (d.cut == CUT_HALF) return count / 2;
    // The swap loop, 32 positions at a time: the flags of a run are taken
    // before its swaps (independent loads), which is exact because the loop
    // only swaps positions at or before the one it stands on, so a position
    // still holds its first slot when the loop reaches it.
    uint32_t m = 0;
    for (uint32_t base = 0; base < count; base += 32) {
        const uint32_t run = count - base < 32u ? count - base : 32u;
        uint32_t flags = 0;
#pragma unroll 8
        for (uint32_t e = 0; e < run; e++)
            if (bin_of(centres + 3 * (uint64_t)slots[base + e], lo, scale, (int)d.axis) <= d.at) flags |= 1u << e;
        for (uint32_t e = 0; e < run; e++) {
            if ((flags >> e) & 1u) {
                const uint32_t j = base + e;
                const uint32_t t = slots[j];
                slots[j] = slots[m];
                slots[m] = t;
                m++;
            }
        }
    }
    return (m == 0 || m == count) ? count / 2 : m;
}

// One node of the tree under construction (temporary numbering).
struct TNode {
    uint32_t start, end, depth;
    uint32_t left, right;  // temporary ids of the children; NONE for a leaf
};

// Where to put new nodes: a counter of temporary ids and the next level's
// list. `add` is an atomic add on the device and a plain one on the host.
template <class Add>
SAH_HD void process(uint32_t t, TNode* tn, const float* prims, const float* centres, uint32_t* order, uint32_t leaf,
                    uint32_t* tcount, uint32_t* next, uint32_t* next_count, Add add) {
    TNode nd = tn[t];
    const uint32_t m = nd.depth + 1 >= MAX_DEPTH
                           ? NONE
                           : split(prims, centres, order + nd.start, nd.end - nd.start, leaf);
    if (m == NONE) {
        nd.left = nd.right = NONE;
    } else {
        const uint32_t c = add(tcount, 2u);
        tn[c] = TNode{nd.start, nd.start + m, nd.depth + 1, NONE, NONE};
        tn[c + 1] = TNode{nd.start + m, nd.end, nd.depth + 1, NONE, NONE};
        nd.left = c;
        nd.right = c + 1;
        const uint32_t p = add(next_count, 2u);
        next[p] = c;
        next[p + 1] = c + 1;
    }
    tn[t] = nd;
}

// Inner nodes in t's subtree, t included (children's counts first).
SAH_HD void count_inner(uint32_t t, const TNode* tn, uint32_t* inner) {
    const TNode nd = tn[t];
    inner[t] = nd.left == NONE ? 0u : 1u + inner[nd.left] + inner[nd.right];
}

// Top down: an inner node of depth-first rank r has its children at final
// indices 2r + 1 and 2r + 2 (sah.rs:95-105's work stack pops the left child
// first and hands out two indices per inner node).
SAH_HD void place(uint32_t t, const TNode* tn, const uint32_t* inner, uint32_t* rank, uint32_t* final_index) {
    const TNode nd = tn[t];
    if (nd.left == NONE) return;
    const uint32_t r = rank[t];
    rank[nd.left] = r + 1;
    rank[nd.right] = r + 1 + inner[nd.left];
    final_index[nd.left] = 2 * r + 1;
    final_index[nd.right] = 2 * r + 2;
}

// The node at its final index, bounds from its children or its primitives
// (Bvh::refit, build.rs:180-194: unions, exact in any order). `boxes` holds
// each temporary node's bounds for its parent; children come first.
SAH_HD void emit(uint32_t t, const TNode* tn, const uint32_t* final_index, const float* prims, const uint32_t* order,
                 Box* boxes, float* nodes) {
    const TNode nd = tn[t];
    Box b = empty_box();
    uint32_t lo_i, hi_i;
    if (nd.left == NONE) {
        for (uint32_t s = nd.start; s < nd.end; s++) grow(b, prim_box(prims + 8 * (uint64_t)order[s]));
        lo_i = nd.start | LEAF_BIT;
        hi_i = nd.end;
    } else {
        b = boxes[nd.left];
        grow(b, boxes[nd.right]);
        lo_i = final_index[nd.left];
        hi_i = final_index[nd.right];
    }
    boxes[t] = b;
    float* o = nodes + 8 * (uint64_t)final_index[t];
    uint32_t* u = (uint32_t*)o;
    o[0] = b.lo[0];
    o[1] = b.lo[1];
    o[2] = b.lo[2];
    u[3] = lo_i;
    o[4] = b.hi[0];
    o[5] = b.hi[1];
    o[6] = b.hi[2];
    u[7] = hi_i;
}

}  // namespace sah
}  // namespace phx
