// ORACLE — test infrastructure only (see oracle.h). CPU restatement of
// phiray's LBVH builder: src/bvh/node.rs, src/bvh/mod.rs, src/bvh/build.rs,
// src/bvh/shape.rs, and the radix model test in src/bvh/sort.rs.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const uint32_t LEAF = 0x80000000u;  // node.rs:7
const uint32_t STACK = 32;          // node.rs:6

// Rust f32::min / f32::max: the non-NaN argument wins.
inline float rmin(float a, float b) {
    if (a != a) return b;
    if (b != b) return a;
    return a < b ? a : b;
}
inline float rmax(float a, float b) {
    if (a != a) return b;
    if (b != b) return a;
    return a > b ? a : b;
}

// Aabb::default (node.rs:68-72): lo = f32::MAX, hi = f32::MIN.
inline orc_aabb aabb_default() {
    orc_aabb a;
    std::memset(&a, 0, sizeof a);
    for (int k = 0; k < 3; k++) {
        a.lo[k] = FLT_MAX;
        a.hi[k] = -FLT_MAX;
    }
    return a;
}

// Aabb::union (node.rs:83-85).
inline orc_aabb aabb_union(const orc_aabb& a, const orc_aabb& b) {
    orc_aabb r;
    std::memset(&r, 0, sizeof r);
    for (int k = 0; k < 3; k++) {
        r.lo[k] = rmin(a.lo[k], b.lo[k]);
        r.hi[k] = rmax(a.hi[k], b.hi[k]);
    }
    return r;
}

inline uint32_t clz32(uint32_t x) { return x == 0 ? 32u : (uint32_t)__builtin_clz(x); }

// morton's spread (node.rs:98-104): Rust `as u64` of a clamped f32 (NaN
// clamps to NaN and converts to 0).
inline uint64_t spread(float v) {
    if (v != v) return 0;
    float c = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    float s = c * 1023.0f;
    uint64_t x = (uint64_t)s;
    x = (x | (x << 16)) & 0x030000FFull;
    x = (x | (x << 8)) & 0x0300F00Full;
    x = (x | (x << 4)) & 0x030C30C3ull;
    return (x | (x << 2)) & 0x09249249ull;
}

inline orc_node node_inner(uint32_t left, uint32_t right) {
    orc_node n;
    std::memset(&n, 0, sizeof n);
    n.lo.i = left;
    n.hi.i = right;
    return n;
}

inline orc_node node_leaf(uint32_t start, uint32_t end) {
    orc_node n;
    std::memset(&n, 0, sizeof n);
    n.lo.i = start | LEAF;
    n.hi.i = end;
    return n;
}

inline bool is_leaf(const orc_node& n) { return (n.lo.i & LEAF) != 0; }

orc_link link_of(const uint32_t* codes, uint32_t nn, uint32_t ii) {
    // build.rs:28-60
    const int64_t i = ii, n = nn;
    auto delta = [&](int64_t a, int64_t b) { return orc_delta(codes, nn, a, b); };
    const int64_t d = (delta(i, i + 1) - delta(i, i - 1) > 0) ? 1 : -1;
    const int32_t dmin = delta(i, i - d);
    int64_t lmax = 2;
    while (delta(i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0, t = lmax / 2;
    while (t >= 1) {
        if (delta(i, i + (l + t) * d) > dmin) l += t;
        t /= 2;
    }
    const int64_t j = i + l * d;
    const int32_t dnode = delta(i, j);
    int64_t s = 0;
    t = l;
    for (;;) {
        t = (t + 1) >> 1;
        if (delta(i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int64_t g = i + s * d + std::min<int64_t>(d, 0);
    const int64_t first = std::min(i, j), last = std::max(i, j);
    const int64_t left = (first == g) ? n - 1 + g : g;
    const int64_t right = (last == g + 1) ? n + g : g + 1;
    orc_link k;
    k.left = (uint32_t)left;
    k.right = (uint32_t)right;
    k.first = (uint32_t)first;
    k.last = (uint32_t)last;
    return k;
}

}  // namespace

extern "C" {

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

uint64_t orc_morton(const float p[3], uint32_t group) {
    return ((uint64_t)group << 32) | (spread(p[0]) << 2) | (spread(p[1]) << 1) | spread(p[2]);
}

void orc_scene(const orc_aabb* prims, uint32_t n, orc_aabb* out) {
    // build.rs:70-72, a fold from Aabb::default.
    orc_aabb s = aabb_default();
    for (uint32_t i = 0; i < n; i++) s = aabb_union(s, prims[i]);
    *out = s;
}

void orc_codes(const orc_aabb* prims, uint32_t n, uint32_t* codes) {
    // build.rs:75-85
    orc_aabb s;
    orc_scene(prims, n, &s);
    float inv[3];
    for (int k = 0; k < 3; k++) {
        const float e = s.hi[k] - s.lo[k];
        inv[k] = e > 0.0f ? 1.0f / e : 0.0f;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        float u[3];
        for (int k = 0; k < 3; k++) {
            const float c = 0.5f * (prims[i].lo[k] + prims[i].hi[k]);  // Aabb::center
            u[k] = (c - s.lo[k]) * inv[k];
        }
        codes[i] = (uint32_t)orc_morton(u, 0);  // mod.rs:28-30 code()
    }
}

void orc_sort_codes(const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted) {
    // build.rs:87-92: par_sort_unstable_by_key(|&i| (codes[i], i)) is a total
    // order, so any correct sort on that key gives the same result.
    std::vector<uint64_t> key(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) key[i] = ((uint64_t)codes[i] << 32) | (uint64_t)i;
    std::sort(key.begin(), key.end());
    for (uint32_t i = 0; i < n; i++) {
        order[i] = (uint32_t)key[i];
        sorted[i] = (uint32_t)(key[i] >> 32);
    }
}

void orc_radix_model(const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted) {
    // sort.rs:127-150: key = [index, code]; digit d reads the index word for
    // shifts below 32, the code word above; a histogram, an exclusive prefix
    // and a sequential scatter per pass.
    const uint32_t DIGIT = 8, PASSES = 8, BINS = 256;
    std::vector<uint32_t> k0(n), k1(n), a0(n), a1(n);
    for (uint32_t i = 0; i < n; i++) {
        k0[i] = i;
        k1[i] = codes[i];
    }
    for (uint32_t d = 0; d < PASSES; d++) {
        const uint32_t shift = d * DIGIT;
        auto digit = [&](uint32_t i) {
            return shift < 32 ? (k0[i] >> shift) & 0xFF : (k1[i] >> (shift - 32)) & 0xFF;
        };
        std::vector<uint32_t> cursor(BINS, 0);
        for (uint32_t i = 0; i < n; i++) cursor[digit(i)]++;
        uint32_t running = 0;
        for (uint32_t b = 0; b < BINS; b++) {
            const uint32_t c = cursor[b];
            cursor[b] = running;
            running += c;
        }
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t b = digit(i);
            a0[cursor[b]] = k0[i];
            a1[cursor[b]] = k1[i];
            cursor[b]++;
        }
        std::swap(k0, a0);
        std::swap(k1, a1);
    }
    for (uint32_t i = 0; i < n; i++) {
        order[i] = k0[i];
        sorted[i] = k1[i];
    }
}

int32_t orc_delta(const uint32_t* codes, uint32_t n, int64_t i, int64_t j) {
    // mod.rs:33-43
    if (j < 0 || j >= (int64_t)n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a != b) return (int32_t)clz32(a ^ b);
    return 32 + (int32_t)clz32((uint32_t)i ^ (uint32_t)j);
}

void orc_links(const uint32_t* sorted, uint32_t n, orc_link* links) {
    // build.rs:97 (rayon over internal nodes).
    if (n < 2) return;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n - 1; i++) links[i] = link_of(sorted, n, (uint32_t)i);
}

void orc_assemble(uint32_t n, const orc_link* links, uint32_t leaf, orc_node* nodes, uint32_t* depth_out) {
    // build.rs:139-168 (serial DFS, as in the reference).
    *depth_out = 0;
    if (n == 0) return;
    for (uint32_t i = 0; i + 1 < n; i++) nodes[i] = node_inner(links[i].left, links[i].right);
    for (uint32_t k = 0; k < n; k++) nodes[n - 1 + k] = node_leaf(k, k + 1);
    uint32_t depth = 0;
    std::vector<std::pair<uint32_t, uint32_t>> stack;
    stack.push_back({0, 0});
    while (!stack.empty()) {
        auto [i, d] = stack.back();
        stack.pop_back();
        depth = std::max(depth, d);
        if (i >= n - 1) continue;
        const orc_link& l = links[i];
        if (l.last - l.first < leaf || d + 1 >= STACK) {
            nodes[i].lo.i = l.first | LEAF;
            nodes[i].hi.i = l.last + 1;
            continue;
        }
        stack.push_back({l.left, d + 1});
        stack.push_back({l.right, d + 1});
    }
    *depth_out = depth;
}

void orc_refit(orc_node* nodes, uint32_t nnodes, const uint32_t* order, const orc_aabb* prims) {
    // build.rs:180-194: iterative post-order from the root.
    if (nnodes == 0) return;
    std::vector<std::pair<uint32_t, bool>> stack;
    stack.push_back({0, false});
    while (!stack.empty()) {
        auto [i, done] = stack.back();
        stack.pop_back();
        const orc_node nd = nodes[i];
        orc_aabb b;
        if (is_leaf(nd)) {
            b = aabb_default();
            for (uint32_t s = nd.lo.i & ~LEAF; s < nd.hi.i; s++) b = aabb_union(b, prims[order[s]]);
        } else if (done) {
            orc_aabb l, r;
            std::memset(&l, 0, sizeof l);
            std::memset(&r, 0, sizeof r);
            const orc_node& a = nodes[nd.lo.i & ~LEAF];
            const orc_node& c = nodes[nd.hi.i & ~LEAF];
            for (int k = 0; k < 3; k++) {
                l.lo[k] = a.lo.p[k];
                l.hi[k] = a.hi.p[k];
                r.lo[k] = c.lo.p[k];
                r.hi[k] = c.hi.p[k];
            }
            b = aabb_union(l, r);
        } else {
            stack.push_back({i, true});
            stack.push_back({nd.lo.i & ~LEAF, false});
            stack.push_back({nd.hi.i & ~LEAF, false});
            continue;
        }
        for (int k = 0; k < 3; k++) {
            nodes[i].lo.p[k] = b.lo[k];
            nodes[i].hi.p[k] = b.hi[k];
        }
    }
}

// ---- the binned SAH builder (src/bvh/sah.rs:25-189): the tree phiray's
// tracer walks (forest.rs:49, 216). Bins, sweeps and the in-place partition
// in the reference's order, so the tree is the reference's node for node.
namespace {

const uint32_t SAH_BINS = 16;      // sah.rs:26 BIN_COUNT
const float SAH_TRAVERSE = 1.0f;   // sah.rs:30 TRAVERSE

// sah.rs:32-35 area (of an Aabb; negative extents count as 0).
float sah_area(const orc_aabb& b) {
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = rmax(b.hi[k] - b.lo[k], 0.0f);
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
}

// sah.rs:68-79 Grid: a centroid's bin along one axis (Rust `as usize`
// truncates and saturates; NaN gives 0).
struct SahGrid {
    float lo[3], scale[3];
    uint32_t bin(const float* c, int k) const {
        const float v = (c[k] - lo[k]) * scale[k];
        uint64_t b = (v != v || v <= 0.0f) ? 0u : (v >= 1.8e19f ? UINT64_MAX : (uint64_t)v);
        return (uint32_t)std::min<uint64_t>(b, SAH_BINS - 1);
    }
};

orc_aabb point_box(const float* c) {
    orc_aabb b;
    std::memset(&b, 0, sizeof b);
    for (int k = 0; k < 3; k++) b.lo[k] = b.hi[k] = c[k];
    return b;
}

// sah.rs:114-189 split: the left count m after reordering `slots`, or -1
// for a leaf. Histogram merges are exact (integer counts, min/max bounds),
// so the reference's parallel fill gives what this serial one gives.
int64_t sah_split(const orc_aabb* prims, const std::vector<float>& centres, uint32_t* slots, uint32_t count,
                  uint32_t leaf) {
    if (count <= 1) return -1;
    orc_aabb cbox = aabb_default();
    for (uint32_t j = 0; j < count; j++) cbox = aabb_union(cbox, point_box(&centres[3 * (size_t)slots[j]]));
    SahGrid grid;
    bool flat = true;
    for (int k = 0; k < 3; k++) {
        const float e = cbox.hi[k] - cbox.lo[k];
        grid.lo[k] = cbox.lo[k];
        grid.scale[k] = e > 0.0f ? (float)SAH_BINS * (1.0f - 1e-5f) / e : 0.0f;
        if (grid.scale[k] != 0.0f) flat = false;
    }
    if (flat) return count > leaf ? (int64_t)(count / 2) : -1;
    uint32_t bcount[3][SAH_BINS] = {};
    orc_aabb bbox[3][SAH_BINS];
    for (int k = 0; k < 3; k++)
        for (uint32_t b = 0; b < SAH_BINS; b++) bbox[k][b] = aabb_default();
    for (uint32_t j = 0; j < count; j++) {
        const uint32_t i = slots[j];
        for (int k = 0; k < 3; k++) {
            const uint32_t at = grid.bin(&centres[3 * (size_t)i], k);
            bcount[k][at] += 1;
            bbox[k][at] = aabb_union(bbox[k][at], prims[i]);
        }
    }
    bool have = false;
    float best_cost = 0.0f;
    int best_k = 0;
    uint32_t best_at = 0;
    for (int k = 0; k < 3; k++) {
        if (grid.scale[k] == 0.0f) continue;
        float right_area[SAH_BINS] = {};
        uint32_t right_count[SAH_BINS] = {};
        orc_aabb b = aabb_default();
        uint32_t c = 0;
        for (uint32_t at = SAH_BINS - 1; at >= 1; at--) {
            b = aabb_union(b, bbox[k][at]);
            c += bcount[k][at];
            right_area[at] = sah_area(b);
            right_count[at] = c;
        }
        b = aabb_default();
        c = 0;
        for (uint32_t at = 0; at + 1 < SAH_BINS; at++) {
            b = aabb_union(b, bbox[k][at]);
            c += bcount[k][at];
            const float ra = right_area[at + 1];
            const uint32_t rc = right_count[at + 1];
            if (c == 0 || rc == 0) continue;
            const float cost = sah_area(b) * (float)c + ra * (float)rc;
            if (!have || cost < best_cost) {
                have = true;
                best_cost = cost;
                best_k = k;
                best_at = at;
            }
        }
    }
    orc_aabb bounds = aabb_default();
    for (uint32_t b = 0; b < SAH_BINS; b++) bounds = aabb_union(bounds, bbox[0][b]);
    if (!have) return count > leaf ? (int64_t)(count / 2) : -1;
    const float parent = rmax(sah_area(bounds), FLT_MIN);
    if (count <= leaf && SAH_TRAVERSE + best_cost / parent >= (float)count) return -1;
    uint32_t m = 0;
    for (uint32_t j = 0; j < count; j++) {
        if (grid.bin(&centres[3 * (size_t)slots[j]], best_k) <= best_at) {
            std::swap(slots[j], slots[m]);
            m++;
        }
    }
    return (m == 0 || m == count) ? (int64_t)(count / 2) : (int64_t)m;
}

}  // namespace

uint32_t orc_build_sah(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* nodes, uint32_t* order,
                       uint32_t* depth_out) {
    // sah.rs:84-109 Bvh::build_sah: a work stack of (slot, start, end, depth),
    // left child taken first, leaves at the depth cap, then refit.
    *depth_out = 0;
    if (n == 0) return 0;
    std::vector<float> centres(3 * (size_t)n);
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) centres[3 * (size_t)i + k] = 0.5f * (prims[i].lo[k] + prims[i].hi[k]);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    uint32_t count = 1;
    nodes[0] = node_inner(0, 0);
    uint32_t depth = 0;
    struct Work {
        uint32_t slot, start, end, d;
    };
    std::vector<Work> work{{0, 0, n, 0}};
    while (!work.empty()) {
        const Work wk = work.back();
        work.pop_back();
        depth = std::max(depth, wk.d);
        const int64_t cut = wk.d + 1 >= STACK ? -1 : sah_split(prims, centres, order + wk.start, wk.end - wk.start, leaf);
        if (cut < 0) {
            nodes[wk.slot] = node_leaf(wk.start, wk.end);
        } else {
            const uint32_t at = count;
            nodes[count++] = node_inner(0, 0);
            nodes[count++] = node_inner(0, 0);
            nodes[wk.slot] = node_inner(at, at + 1);
            const uint32_t m = (uint32_t)cut;
            work.push_back({at + 1, wk.start + m, wk.end, wk.d + 1});
            work.push_back({at, wk.start, wk.start + m, wk.d + 1});
        }
    }
    *depth_out = depth;
    orc_refit(nodes, count, order, prims);
    return count;
}

void orc_build(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* nodes, uint32_t* order, uint32_t* depth) {
    // build.rs:94-100
    *depth = 0;
    if (n == 0) return;
    std::vector<uint32_t> codes(n), sorted(n);
    orc_codes(prims, n, codes.data());
    orc_sort_codes(codes.data(), n, order, sorted.data());
    std::vector<orc_link> links(n > 1 ? n - 1 : 0);
    orc_links(sorted.data(), n, links.data());
    orc_assemble(n, links.data(), leaf, nodes, depth);
    orc_refit(nodes, 2 * n - 1, order, prims);
}

uint32_t orc_build_compact(const orc_aabb* prims, uint32_t n, uint32_t leaf, orc_node* out, uint32_t* order,
                           uint32_t* depth_out) {
    // build.rs:104-136: breadth-first, never holding 2n-1 nodes.
    *depth_out = 0;
    if (n == 0) return 0;
    std::vector<uint32_t> codes(n), sorted(n);
    orc_codes(prims, n, codes.data());
    orc_sort_codes(codes.data(), n, order, sorted.data());
    std::vector<orc_link> links(n > 1 ? n - 1 : 0);
    orc_links(sorted.data(), n, links.data());
    std::vector<orc_node> nodes(1, node_inner(0, 0));
    struct Item {
        uint32_t i, slot, d;
    };
    std::deque<Item> queue;
    queue.push_back({0, 0, 0});
    uint32_t depth = 0;
    while (!queue.empty()) {
        Item it = queue.front();
        queue.pop_front();
        depth = std::max(depth, it.d);
        if (it.i >= n - 1) {
            const uint32_t k = it.i - (n - 1);
            nodes[it.slot] = node_leaf(k, k + 1);
            continue;
        }
        const orc_link& l = links[it.i];
        if (l.last - l.first < leaf || it.d + 1 >= STACK) {
            nodes[it.slot] = node_leaf(l.first, l.last + 1);
            continue;
        }
        const uint32_t at = (uint32_t)nodes.size();
        nodes.push_back(node_inner(0, 0));
        nodes.push_back(node_inner(0, 0));
        nodes[it.slot] = node_inner(at, at + 1);
        queue.push_back({l.left, at, it.d + 1});
        queue.push_back({l.right, at + 1, it.d + 1});
    }
    orc_refit(nodes.data(), (uint32_t)nodes.size(), order, prims);
    std::memcpy(out, nodes.data(), nodes.size() * sizeof(orc_node));
    *depth_out = depth;
    return (uint32_t)nodes.size();
}

uint32_t orc_compact(orc_node* nodes, uint32_t nnodes) {
    // shape.rs:8-37
    if (nnodes == 0) return 0;
    std::vector<uint32_t> map(nnodes, 0xFFFFFFFFu);
    std::vector<uint32_t> keep(1, 0);
    map[0] = 0;
    for (size_t i = 0; i < keep.size(); i++) {
        const orc_node nd = nodes[keep[i]];
        if (!is_leaf(nd)) {
            for (uint32_t c : {nd.lo.i & ~LEAF, nd.hi.i & ~LEAF}) {
                map[c] = (uint32_t)keep.size();
                keep.push_back(c);
            }
        }
    }
    std::vector<orc_node> out;
    out.reserve(keep.size());
    for (uint32_t k : keep) {
        orc_node nd = nodes[k];
        if (!is_leaf(nd)) {
            nd.lo.i = map[nd.lo.i & ~LEAF];
            nd.hi.i = map[nd.hi.i & ~LEAF];
        }
        out.push_back(nd);
    }
    std::memcpy(nodes, out.data(), out.size() * sizeof(orc_node));
    return (uint32_t)out.size();
}

uint32_t orc_reachable(const orc_node* nodes, uint32_t nnodes, uint32_t* out) {
    // shape.rs:40-51
    uint32_t count = 0;
    if (nnodes == 0) return 0;
    std::vector<uint32_t> stack(1, 0);
    while (!stack.empty()) {
        const uint32_t i = stack.back();
        stack.pop_back();
        out[count++] = i;
        const orc_node& nd = nodes[i];
        if (!is_leaf(nd)) {
            stack.push_back(nd.lo.i & ~LEAF);
            stack.push_back(nd.hi.i & ~LEAF);
        }
    }
    return count;
}

}  // extern "C"
