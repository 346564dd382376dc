// The Rendered-mode tracer (phiray Tracer, src/trace/*.rs) on the device.
//
// A scene is uploaded once; its LBVH is built on the device over the face
// boxes (bvh.cu) and re-encoded for the walk (shade.cuh): inner nodes with
// both children's boxes inline, triangles gathered into leaf order. The
// sample kernel runs shade.wgsl's main for every pixel and keeps the
// per-pixel sums in registers across all the samples of a call, writing the
// image planes once at the end — the same sums, in the same order, that the
// reference's one-dispatch-per-sample loop leaves in its px buffer.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <memory>
#include <cstring>
#include <vector>

#include "lbvh.cuh"
#include "render.cuh"

namespace phx {

using namespace shade;

namespace {

// ---- scene preparation ----

// The scene checks Tracer::new's callers rely on, run over the uploaded
// arrays before any kernel indexes through them: out[0] the first face that
// names a vertex or material out of range, out[1] the first material with a
// texture or map (Mat words 12-16 not NO_TEX), out[2] the first with a
// second lobe (word 30 not NO_MAT), all 0xFFFFFFFF when none; out[3] != 0
// when some material emits (luminance of words 8-10 above zero).
__global__ void __launch_bounds__(256) k_check_scene(const uint4* __restrict__ faces, uint32_t nfaces, uint32_t nverts,
                                                     const float* __restrict__ mats, uint32_t nmats,
                                                     uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nfaces) {
        const uint4 q = __ldg(faces + i);
        if (q.x >= nverts || q.y >= nverts || q.z >= nverts || q.w >= nmats) atomicMin(out, i);
    }
    if (i < nmats) {
        const float* m = mats + 32 * (size_t)i;
        const uint32_t* w = (const uint32_t*)m;
        bool tex = false;
        for (int k = 12; k <= 16; k++) tex = tex || __ldg(w + k) != 0xFFFFFFFFu;
        if (tex) atomicMin(out + 1, i);
        if (__ldg(w + 30) != 0xFFFFFFFFu) atomicMin(out + 2, i);
        if (0.2126f * __ldg(m + 8) + 0.7152f * __ldg(m + 9) + 0.0722f * __ldg(m + 10) > 0.0f) atomicOr(out + 3, 1u);
    }
}

// tris in slot order (sorted by Morton code): positions, face id, material,
// and the shadow-pass flag from the material (bvh.wgsl:158-162).
__global__ void k_gather(const uint32_t* __restrict__ order, const uint4* __restrict__ faces,
                         const float4* __restrict__ verts, const float4* __restrict__ vnorm,
                         const float4* __restrict__ mats, uint32_t nmats, uint32_t n, float4* __restrict__ tris,
                         float4* __restrict__ tnorm, uint32_t* status) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t f = __ldg(order + s);
    const uint4 v = __ldg(faces + f);
    const float4 a = __ldg(verts + v.x), b = __ldg(verts + v.y), c = __ldg(verts + v.z);
    uint32_t m = v.w;
    if (m >= nmats) {
        atomicOr(status, STATUS_BAD_INDEX);
        m = 0;
    }
    const float4 m0 = __ldg(mats + 8 * (size_t)m), m1 = __ldg(mats + 8 * (size_t)m + 1);
    const uint32_t flags = (m1.z > 0.5f || m0.w < 0.5f) ? FLAG_PASS : 0u;
    tris[3 * (size_t)s] = make_float4(a.x, a.y, a.z, __uint_as_float(f));
    tris[3 * (size_t)s + 1] = make_float4(b.x, b.y, b.z, __uint_as_float(m));
    tris[3 * (size_t)s + 2] = make_float4(c.x, c.y, c.z, __uint_as_float(flags));
    if (tnorm) {
        tnorm[3 * (size_t)s] = __ldg(vnorm + v.x);
        tnorm[3 * (size_t)s + 1] = __ldg(vnorm + v.y);
        tnorm[3 * (size_t)s + 2] = __ldg(vnorm + v.z);
    }
}

// Marks the last slot of every reachable leaf (the refit's start list).
__global__ void k_mark_ends(const float4* __restrict__ nodes, const uint32_t* __restrict__ starts,
                            const uint32_t* __restrict__ nstarts, float4* tris) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nstarts) return;
    const uint32_t i = starts[t];
    const uint32_t end = __float_as_uint(nodes[2 * (size_t)i + 1].w);
    float4* c = tris + 3 * (size_t)(end - 1) + 2;
    c->w = __uint_as_float(__float_as_uint(c->w) | FLAG_END);
}

// The refit (k_refit's leaf part and climb) fused with the triangle gather
// for a single-mesh LBVH tree: the thread of each reachable leaf computes
// its faces' boxes from the vertices (Aabb::of_tri, as k_face_boxes), writes
// their slots' triangle records (as k_gather) with the last slot marked (as
// k_mark_ends), stores the leaf's box and climbs. The nodes, triangles and
// flags are those of the separate kernels; the vertices are read once.
__global__ void __launch_bounds__(256) k_refit_gather(const uint32_t* __restrict__ order,
                                                      const uint4* __restrict__ faces,
                                                      const float4* __restrict__ verts,
                                                      const float4* __restrict__ vnorm,
                                                      const float4* __restrict__ mats, uint32_t nmats,
                                                      float4* __restrict__ tris, float4* __restrict__ tnorm,
                                                      const uint32_t* __restrict__ parent, float4* nodes,
                                                      const uint32_t* __restrict__ starts,
                                                      const uint32_t* __restrict__ nstarts, uint32_t* counters,
                                                      uint32_t* status) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nstarts) return;
    const uint32_t i = starts[t];
    const float4 na = nodes[2 * (size_t)i], nb = nodes[2 * (size_t)i + 1];
    const uint32_t first = __float_as_uint(na.w) & ~LEAF, end = __float_as_uint(nb.w);
    float lx = FLT_MAX, ly = FLT_MAX, lz = FLT_MAX, hx = -FLT_MAX, hy = -FLT_MAX, hz = -FLT_MAX;
    for (uint32_t s = first; s < end; s++) {
        const uint32_t f = __ldg(order + s);
        const uint4 v = __ldg(faces + f);
        const float4 a = __ldg(verts + v.x), b = __ldg(verts + v.y), c = __ldg(verts + v.z);
        lx = fminf(lx, fminf(fminf(a.x, b.x), c.x));
        ly = fminf(ly, fminf(fminf(a.y, b.y), c.y));
        lz = fminf(lz, fminf(fminf(a.z, b.z), c.z));
        hx = fmaxf(hx, fmaxf(fmaxf(a.x, b.x), c.x));
        hy = fmaxf(hy, fmaxf(fmaxf(a.y, b.y), c.y));
        hz = fmaxf(hz, fmaxf(fmaxf(a.z, b.z), c.z));
        uint32_t m = v.w;
        if (m >= nmats) {
            atomicOr(status, STATUS_BAD_INDEX);
            m = 0;
        }
        const float4 m0 = __ldg(mats + 8 * (size_t)m), m1 = __ldg(mats + 8 * (size_t)m + 1);
        const uint32_t flags = ((m1.z > 0.5f || m0.w < 0.5f) ? FLAG_PASS : 0u) | (s + 1 == end ? FLAG_END : 0u);
        tris[3 * (size_t)s] = make_float4(a.x, a.y, a.z, __uint_as_float(f));
        tris[3 * (size_t)s + 1] = make_float4(b.x, b.y, b.z, __uint_as_float(m));
        tris[3 * (size_t)s + 2] = make_float4(c.x, c.y, c.z, __uint_as_float(flags));
        if (tnorm) {
            tnorm[3 * (size_t)s] = __ldg(vnorm + v.x);
            tnorm[3 * (size_t)s + 1] = __ldg(vnorm + v.y);
            tnorm[3 * (size_t)s + 2] = __ldg(vnorm + v.z);
        }
    }
    nodes[2 * (size_t)i] = make_float4(lx, ly, lz, na.w);
    nodes[2 * (size_t)i + 1] = make_float4(hx, hy, hz, nb.w);
    refit_climb(i, lx, ly, lz, hx, hy, hz, parent, nodes, counters, status);
}

// Marks the last slot of every leaf of a tree whose nodes are all reachable
// (the binned SAH tree's compact array).
__global__ void k_mark_leaf_ends(const float4* __restrict__ nodes, uint32_t m, float4* tris) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const float4 a = nodes[2 * (size_t)i], b = nodes[2 * (size_t)i + 1];
    if (!(__float_as_uint(a.w) & LEAF)) return;
    const uint32_t end = __float_as_uint(b.w);
    float4* c = tris + 3 * (size_t)(end - 1) + 2;
    c->w = __uint_as_float(__float_as_uint(c->w) | FLAG_END);
}

// A child's ref in the walk's records: an inner node's record index (its
// Karras index + inner_base), or for a leaf its first slot + leaf_base with
// LEAF and leaf_bits (INST for a top-tree leaf).
__device__ __forceinline__ uint32_t child_ref(uint32_t node_word, uint32_t index, uint32_t inner_base,
                                              uint32_t leaf_base, uint32_t leaf_bits) {
    if (node_word & LEAF) return ((node_word & ~LEAF) + leaf_base) | LEAF | leaf_bits;
    return index + inner_base;
}

// Inner node i -> both children's boxes and refs, into record inner_base + i.
__global__ void k_convert(const float4* __restrict__ nodes, uint32_t ninner, float4* __restrict__ out,
                          uint32_t inner_base, uint32_t leaf_base, uint32_t leaf_bits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninner) return;
    const float4 a = nodes[2 * (size_t)i], b = nodes[2 * (size_t)i + 1];
    const uint32_t li = __float_as_uint(a.w), ri = __float_as_uint(b.w);
    if (li & LEAF) return;  // a packed leaf: never walked as an inner node
    const float4 la = nodes[2 * (size_t)li], lb = nodes[2 * (size_t)li + 1];
    const float4 ra = nodes[2 * (size_t)ri], rb = nodes[2 * (size_t)ri + 1];
    const uint32_t lr = child_ref(__float_as_uint(la.w), li, inner_base, leaf_base, leaf_bits);
    const uint32_t rr = child_ref(__float_as_uint(ra.w), ri, inner_base, leaf_base, leaf_bits);
    out += 4 * (size_t)inner_base;
    float4* q = out + 4 * (size_t)i;
    q[0] = make_float4(la.x, la.y, la.z, lb.x);
    q[1] = make_float4(lb.y, lb.z, ra.x, ra.y);
    q[2] = make_float4(ra.z, rb.x, rb.y, rb.z);
    q[3] = make_float4(__uint_as_float(lr), __uint_as_float(rr), 0.0f, 0.0f);
}

// Root box, root ref and the scene extent (Forest::extent, forest.rs:192-200:
// the root box's diagonal, at least 1e-3). leaf_bits: INST for a top tree.
__global__ void k_root(const float4* __restrict__ nodes, uint32_t n, float4* info, uint32_t leaf_bits) {
    const float4 a = nodes[0], b = nodes[1];
    const uint32_t li = __float_as_uint(a.w);
    const uint32_t root = (li & LEAF) ? (li | leaf_bits) : 0u;
    float e = 0.0f;
    const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    e = e + dx * dx;
    e = e + dy * dy;
    e = e + dz * dz;
    const float ext = fmaxf(sqrtf(e), 1e-3f);
    info[0] = make_float4(a.x, a.y, a.z, __uint_as_float(root));
    info[1] = make_float4(b.x, b.y, b.z, ext);
}

// The emitter table (lamp.rs table_of, one instance): emissive slots in slot
// order with their power (world area x emitted luminance) and its running
// share. One block: counts per thread chunk, a block scan for positions,
// then one thread sums in slot order so the CDF rounds as the CPU's does.
__global__ void __launch_bounds__(1024) k_lamps(const float4* __restrict__ tris, const float4* __restrict__ mats,
                                                uint32_t n, uint32_t* __restrict__ slots, float* __restrict__ power,
                                                float* __restrict__ cdf, float4* info) {
    __shared__ uint32_t s_count[1024];
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const uint32_t chunk = (n + T - 1) / T;
    const uint32_t lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
    auto glow = [&](uint32_t s, float& p) -> bool {
        const float4 A = __ldg(tris + 3 * (size_t)s), B = __ldg(tris + 3 * (size_t)s + 1),
                     Cc = __ldg(tris + 3 * (size_t)s + 2);
        const uint32_t m = __float_as_uint(B.w);
        const float4 e = __ldg(mats + 8 * (size_t)m + 2);
        const float lum = 0.2126f * e.x + 0.7152f * e.y + 0.0722f * e.z;
        if (!(lum > 0.0f)) return false;
        const float e1x = B.x - A.x, e1y = B.y - A.y, e1z = B.z - A.z;
        const float e2x = Cc.x - A.x, e2y = Cc.y - A.y, e2z = Cc.z - A.z;
        const float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        float sq = 0.0f;
        sq = sq + cx * cx;
        sq = sq + cy * cy;
        sq = sq + cz * cz;
        p = 0.5f * sqrtf(sq) * lum;
        return p > 0.0f;
    };
    uint32_t c = 0;
    for (uint32_t s = lo; s < hi; s++) {
        float p;
        if (glow(s, p)) c++;
    }
    s_count[t] = c;
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < T; k++) {
            const uint32_t v = s_count[k];
            s_count[k] = run;
            run += v;
        }
        info[2] = make_float4(__uint_as_float(run), 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();
    uint32_t at = s_count[t];
    for (uint32_t s = lo; s < hi; s++) {
        float p;
        if (glow(s, p)) {
            slots[at] = s;
            power[at] = p;
            at++;
        }
    }
    __syncthreads();
    if (t == 0) {
        const uint32_t count = __float_as_uint(info[2].x);
        float total = 0.0f;
        for (uint32_t k = 0; k < count; k++) total += power[k];
        float run = 0.0f;
        for (uint32_t k = 0; k < count; k++) {
            run += power[k];
            cdf[k] = run / total;
        }
    }
}

// ---- scenes of instances (forest.rs, instance.rs, lamp.rs) ----

// slot s of a mesh's range [lo, lo + n) -> the face it holds, from the
// mesh tree's order (Forest::build's order: faces permuted within the range).
__global__ void k_mesh_order(const uint32_t* __restrict__ order, uint32_t n, uint32_t lo, uint32_t* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[lo + s] = lo + order[s];
}

// A mesh's root record (2 float4): its tree's root box, the root's ref
// (record index, or first slot | LEAF), both in the walk's numbering.
__global__ void k_mesh_root(const float4* __restrict__ nodes, float4* __restrict__ rec, uint32_t inner_base,
                            uint32_t leaf_base) {
    const float4 a = nodes[0], b = nodes[1];
    const uint32_t root = child_ref(__float_as_uint(a.w), 0u, inner_base, leaf_base, 0u);
    rec[0] = make_float4(a.x, a.y, a.z, __uint_as_float(root));
    rec[1] = make_float4(b.x, b.y, b.z, 0.0f);
}

// Each instance's mesh root box and ref (words 6 and 7 of its record), with
// its flags; a mesh with no faces has root NONE (never walked).
__global__ void k_inst_fill(float4* __restrict__ rec, const float4* __restrict__ mesh_rec,
                            const uint32_t* __restrict__ mesh_of, const uint32_t* __restrict__ flags, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 lo = mesh_rec[2 * (size_t)mesh_of[i]], hi = mesh_rec[2 * (size_t)mesh_of[i] + 1];
    rec[8 * (size_t)i + 6] = lo;
    rec[8 * (size_t)i + 7] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(flags[i]));
}

// Instance::world_box (instance.rs:118-127): the eight corners of the mesh's
// root box placed in the world, for the placed instances (top-tree prims).
__global__ void k_inst_boxes(const float4* __restrict__ rec, const uint32_t* __restrict__ placed, uint32_t n,
                             phx_aabb* __restrict__ boxes) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4* q = rec + 8 * (size_t)placed[k];
    const float4 r[3] = {q[0], q[1], q[2]};
    const float4 lo = q[6], hi = q[7];
    float bl[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bh[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int c = 0; c < 8; c++) {
        const f3 p = mk((c & 1) == 0 ? lo.x : hi.x, (c & 2) == 0 ? lo.y : hi.y, (c & 4) == 0 ? lo.z : hi.z);
        for (int j = 0; j < 3; j++) {
            const float w = row_point(r[j], p);
            bl[j] = fminf(bl[j], w);
            bh[j] = fmaxf(bh[j], w);
        }
    }
    phx_aabb b;
    b.lo[0] = bl[0], b.lo[1] = bl[1], b.lo[2] = bl[2], b.pad_a = 0.0f;
    b.hi[0] = bh[0], b.hi[1] = bh[1], b.hi[2] = bh[2], b.pad_b = 0.0f;
    boxes[k] = b;
}

// inst_order (forest.rs:119): top slot -> instance.
__global__ void k_inst_slots(const uint32_t* __restrict__ order, const uint32_t* __restrict__ placed, uint32_t n,
                             uint32_t* __restrict__ slots) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) slots[s] = placed[order[s]];
}

// The last slot of every top-tree leaf gets INST_END.
__global__ void k_inst_ends(const float4* __restrict__ nodes, const uint32_t* __restrict__ starts,
                            const uint32_t* __restrict__ nstarts, uint32_t* slots) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nstarts) return;
    const uint32_t end = __float_as_uint(nodes[2 * (size_t)starts[t] + 1].w);
    slots[end - 1] |= INST_END;
}

// lamp.rs table_of with instances: every emissive slot (slot order), once for
// each instance of its mesh (instance order), its power the face's world
// area times the emitted luminance; then the running share. One block:
// counts per thread chunk, a block scan for positions, one thread sums in
// table order so the CDF rounds as the CPU's does.
__global__ void __launch_bounds__(1024) k_lamps_inst(const float4* __restrict__ tris, const float4* __restrict__ mats,
                                                     const float4* __restrict__ rec,
                                                     const uint32_t* __restrict__ slot_mesh,
                                                     const uint32_t* __restrict__ mesh_off,
                                                     const uint32_t* __restrict__ mesh_list, uint32_t n,
                                                     uint32_t* __restrict__ slots, uint32_t* __restrict__ insts,
                                                     float* __restrict__ power, float* __restrict__ cdf, float4* info) {
    __shared__ uint32_t s_count[1024];
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const uint32_t chunk = (n + T - 1) / T;
    const uint32_t lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
    // power of (slot s, instance i), or 0
    auto glow = [&](uint32_t s, uint32_t i) -> float {
        const float4 A = __ldg(tris + 3 * (size_t)s), B = __ldg(tris + 3 * (size_t)s + 1),
                     Cc = __ldg(tris + 3 * (size_t)s + 2);
        const uint32_t m = __float_as_uint(B.w);
        const float4 e = __ldg(mats + 8 * (size_t)m + 2);
        const float lum = 0.2126f * e.x + 0.7152f * e.y + 0.0722f * e.z;
        if (!(lum > 0.0f)) return 0.0f;
        const float4* q = rec + 8 * (size_t)i;
        const float4 r0 = q[0], r1 = q[1], r2 = q[2];
        const f3 a = mk(row_point(r0, xyz(A)), row_point(r1, xyz(A)), row_point(r2, xyz(A)));
        const f3 b = mk(row_point(r0, xyz(B)), row_point(r1, xyz(B)), row_point(r2, xyz(B)));
        const f3 c = mk(row_point(r0, xyz(Cc)), row_point(r1, xyz(Cc)), row_point(r2, xyz(Cc)));
        const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
        const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
        const float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        float sq = 0.0f;
        sq = sq + cx * cx;
        sq = sq + cy * cy;
        sq = sq + cz * cz;
        const float p = 0.5f * sqrtf(sq) * lum;
        return p > 0.0f ? p : 0.0f;
    };
    uint32_t c = 0;
    for (uint32_t s = lo; s < hi; s++) {
        const uint32_t k = slot_mesh[s];
        if (k == NONE) continue;
        for (uint32_t j = mesh_off[k]; j < mesh_off[k + 1]; j++)
            if (glow(s, mesh_list[j]) > 0.0f) c++;
    }
    s_count[t] = c;
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < T; k++) {
            const uint32_t v = s_count[k];
            s_count[k] = run;
            run += v;
        }
        info[2] = make_float4(__uint_as_float(run), 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();
    uint32_t at = s_count[t];
    for (uint32_t s = lo; s < hi; s++) {
        const uint32_t k = slot_mesh[s];
        if (k == NONE) continue;
        for (uint32_t j = mesh_off[k]; j < mesh_off[k + 1]; j++) {
            const float p = glow(s, mesh_list[j]);
            if (p > 0.0f) {
                slots[at] = s;
                insts[at] = mesh_list[j];
                power[at] = p;
                at++;
            }
        }
    }
    __syncthreads();
    if (t == 0) {
        const uint32_t count = __float_as_uint(info[2].x);
        float total = 0.0f;
        for (uint32_t k = 0; k < count; k++) total += power[k];
        float run = 0.0f;
        for (uint32_t k = 0; k < count; k++) {
            run += power[k];
            cdf[k] = run / total;
        }
    }
}

// Primary ray of each pixel: face id and t (a warp's pixels an 8 x 4 tile
// where the frame's sides allow, as in k_render).
__global__ void k_primary(Scene S, Frame F, uint32_t frame, uint32_t* __restrict__ ids, float* __restrict__ ts) {
    setup(S, F);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= F.n) return;
    const uint32_t i = tile_px(F, k, 0u, F.n);
    uint32_t seed = hash(i * 9781u + frame * 6271u + 1u);
    const CamRay cr = camera_ray(F, i, seed);
    Count cnt{0, 0, 0};
    const Hit h = walk_scene<false>(S, cr.o, cr.d, INF, false, cnt);
    ids[i] = h.tri == NONE ? NONE : __float_as_uint(__ldg(S.tris + 3 * (size_t)h.tri).w);
    ts[i] = h.t;
}

// One cosine-sampled ray per primary hit (the incoherent set).
__global__ void k_secondary(Scene S, Frame F, uint32_t frame, float4* __restrict__ rays) {
    setup(S, F);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.n) return;
    uint32_t seed = hash(i * 9781u + frame * 6271u + 1u);
    const CamRay cr = camera_ray(F, i, seed);
    Count cnt{0, 0, 0};
    const Hit h = walk_scene<false>(S, cr.o, cr.d, INF, false, cnt);
    if (h.tri == NONE) {
        rays[2 * (size_t)i] = make_float4(cr.o.x, cr.o.y, cr.o.z, 0.0f);
        rays[2 * (size_t)i + 1] = make_float4(cr.d.x, cr.d.y, cr.d.z, 0.0f);
        return;
    }
    const Geo g = geo_at<MODE_ANY>(S, h.tri, h.inst);
    const f3 ng0 = normalize(cross(g.b - g.a, g.c - g.a));
    const f3 ng = dot(ng0, cr.d) < 0.0f ? ng0 : -ng0;
    const f3 pos = cr.o + cr.d * h.t + ng * hit_lift(F, h.t);
    const f3 dir = cosine_dir(ng, seed);
    rays[2 * (size_t)i] = make_float4(pos.x, pos.y, pos.z, INF);
    rays[2 * (size_t)i + 1] = make_float4(dir.x, dir.y, dir.z, 0.0f);
}

template <bool ANY, bool STATS, int P>
__global__ void __launch_bounds__(128) k_rays(Scene S, const float4* __restrict__ rays, uint32_t n,
                                              float4* __restrict__ hits, unsigned long long* counters) {
    __shared__ uint32_t s_stack[P == PLACE_SHARED ? STACK * 128 : 1];
    load_info(S);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count cnt{0, 0, 0};
    if (i < n) {
        const float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
        const Hit h = walk_scene<STATS, P>(S, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, ANY, cnt,
                                              s_stack + threadIdx.x, 128);
        const uint32_t face = h.tri == NONE ? NONE : __float_as_uint(__ldg(S.tris + 3 * (size_t)h.tri).w);
        hits[i] = make_float4(h.t, __uint_as_float(face), h.u, h.v);
    }
    if (STATS) {
        const uint32_t st = __reduce_add_sync(0xffffffffu, cnt.steps);
        const uint32_t te = __reduce_add_sync(0xffffffffu, cnt.tests);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(counters + 1, (unsigned long long)st);
            atomicAdd(counters + 2, (unsigned long long)te);
        }
    }
}

// The same walks on persistent warps that refill idle lanes: every lane
// keeps one ray's traversal state (position in the tree, its 32-entry stack,
// best hit) and advances it STEPS node or leaf visits at a time; between
// rounds the lanes whose ray finished take the next rays from one counter
// (one atomic per warp). Each ray is walked in exactly its own order, so the
// hits are those of k_rays; the warp no longer idles while its longest ray
// finishes.
constexpr int RAY_STEPS = 16;

template <bool ANY, bool STATS>
__global__ void __launch_bounds__(128) k_rays_fetch(Scene S, const float4* __restrict__ rays, uint32_t n,
                                                    float4* __restrict__ hits, unsigned long long* counters,
                                                    uint32_t* next, const uint32_t* __restrict__ order) {
    load_info(S);
    const Tree T = tree_of(S);
    const int lane = threadIdx.x & 31;
    Count cnt{0, 0, 0};
    uint32_t stack[STACK];
    bool active = false;
    uint32_t idx = 0, nd = 0;
    int sp = 0;
    f3 o = mk(0.0f), inv = mk(0.0f);
    RaySpace rs;
    rs.kz = 2u;
    rs.flip = false;
    rs.s = mk(0.0f);
    Hit best{0.0f, NONE, 0.0f, 0.0f};
    for (;;) {
        const uint32_t need = __ballot_sync(0xffffffffu, !active);
        if (need) {
            const int leader = __ffs(need) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next, (uint32_t)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active) {
                idx = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
                if (idx < n) {
                    if (order) idx = __ldg(order + idx);  // walk in the sorted order, answer in place
                    const float4 a = __ldg(rays + 2 * (size_t)idx), b = __ldg(rays + 2 * (size_t)idx + 1);
                    o = mk(a.x, a.y, a.z);
                    const f3 d = mk(b.x, b.y, b.z);
                    cnt.rays++;
                    best = Hit{a.w, NONE, 0.0f, 0.0f};
                    inv = safe_inv(d);
                    rs = ray_space(d);
                    sp = 0;
                    nd = T.root;
                    active = box_t(T.root_lo, T.root_hi, o, inv, best.t) < INF;
                    if (!active) {
                        hits[idx] = make_float4(best.t, __uint_as_float(NONE), 0.0f, 0.0f);
                    }
                    // a ray that misses the root box is written and the lane asks again next round
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            // nothing in flight: done once the counter has passed n
            uint32_t seen = 0;
            if (lane == 0) seen = atomicAdd(next, 0u);
            seen = __shfl_sync(0xffffffffu, seen, 0);
            if (seen >= n) break;
            continue;
        }
        for (int it = 0; it < RAY_STEPS && active; it++) {
            bool done = false;
            if (nd & LEAF) {
                for (uint32_t id = nd & ~LEAF; id < T.nslots; id++) {
                    const float4 A = __ldg(T.tris + 3 * (size_t)id);
                    const float4 B = __ldg(T.tris + 3 * (size_t)id + 1);
                    const float4 Cc = __ldg(T.tris + 3 * (size_t)id + 2);
                    const uint32_t flags = __float_as_uint(Cc.w);
                    if (STATS) cnt.tests++;
                    float u, v;
                    const float t = tri_t(xyz(A), xyz(B), xyz(Cc), o, rs, u, v);
                    if (t < best.t) {
                        if (ANY) {
                            if (!(flags & FLAG_PASS)) {
                                best = Hit{t, id, u, v};
                                done = true;
                                break;
                            }
                        } else {
                            best = Hit{t, id, u, v};
                        }
                    }
                    if (flags & FLAG_END) break;
                }
            } else {
                if (STATS) cnt.steps++;
                const float4* q = T.nodes + 4 * (size_t)nd;
                const float4 n0 = __ldg(q), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3);
                const float tl = box_t(mk(n0.x, n0.y, n0.z), mk(n0.w, n1.x, n1.y), o, inv, best.t);
                const float tr = box_t(mk(n1.z, n1.w, n2.x), mk(n2.y, n2.z, n2.w), o, inv, best.t);
                const uint32_t l = __float_as_uint(n3.x), r = __float_as_uint(n3.y);
                if (tl < INF && tr < INF) {
                    if (sp < STACK) stack[sp++] = tl <= tr ? r : l;
                    nd = tl <= tr ? l : r;
                    continue;
                }
                if (tl < INF) {
                    nd = l;
                    continue;
                }
                if (tr < INF) {
                    nd = r;
                    continue;
                }
            }
            if (!done) {
                if (sp == 0) {
                    done = true;
                } else {
                    sp--;
                    nd = stack[sp];
                }
            }
            if (done) {
                const uint32_t face = best.tri == NONE ? NONE : __float_as_uint(__ldg(T.tris + 3 * (size_t)best.tri).w);
                hits[idx] = make_float4(best.t, __uint_as_float(face), best.u, best.v);
                active = false;
            }
        }
    }
    const uint32_t tot = __reduce_add_sync(0xffffffffu, cnt.rays);
    (void)tot;
    if (STATS) {
        const uint32_t st = __reduce_add_sync(0xffffffffu, cnt.steps);
        const uint32_t te = __reduce_add_sync(0xffffffffu, cnt.tests);
        if (lane == 0) {
            atomicAdd(counters + 1, (unsigned long long)st);
            atomicAdd(counters + 2, (unsigned long long)te);
        }
    }
}

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 9 bits -> every third of 27
    uint32_t x = v & 0x1FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// A ray's sort key: its direction's octant above the 27-bit Morton code of
// its origin in the scene box, so that sorted rays leave nearby points in
// similar directions and walk similar parts of the tree.
__global__ void k_ray_keys(Scene S, const float4* __restrict__ rays, uint32_t n, uint32_t* __restrict__ keys) {
    load_info(S);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
    const f3 ext = S.root_hi - S.root_lo;
    const float ux = ext.x > 0.0f ? (a.x - S.root_lo.x) / ext.x : 0.0f;
    const float uy = ext.y > 0.0f ? (a.y - S.root_lo.y) / ext.y : 0.0f;
    const float uz = ext.z > 0.0f ? (a.z - S.root_lo.z) / ext.z : 0.0f;
    const uint32_t qx = (uint32_t)(fminf(fmaxf(ux, 0.0f), 1.0f) * 511.0f);
    const uint32_t qy = (uint32_t)(fminf(fmaxf(uy, 0.0f), 1.0f) * 511.0f);
    const uint32_t qz = (uint32_t)(fminf(fmaxf(uz, 0.0f), 1.0f) * 511.0f);
    const uint32_t oct = (b.x < 0.0f ? 1u : 0u) | (b.y < 0.0f ? 2u : 0u) | (b.z < 0.0f ? 4u : 0u);
    keys[i] = (oct << 27) | (spread3(qx) << 2) | (spread3(qy) << 1) | spread3(qz);
}

template <bool ANY, bool STATS>
void launch_rays(const Scene& S, const float* rays, uint32_t n, float* hits, unsigned long long* counters,
                 uint32_t place, cudaStream_t s, uint32_t* next = nullptr, int sms = 0, const uint32_t* order = nullptr) {
    if (next && !S.insts) {  // (scenes of instances: a thread per ray)
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rays_fetch<ANY, STATS>, 128, 0);
        const uint32_t grid = std::min<uint32_t>((uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sms, (n + 127) / 128);
        cudaMemsetAsync(next, 0, 4, s);
        k_rays_fetch<ANY, STATS><<<grid, 128, 0, s>>>(S, (const float4*)rays, n, (float4*)hits, counters, next, order);
        return;
    }
    const uint32_t blocks = (n + 127) / 128;
    const float4* r = (const float4*)rays;
    if (place == PHX_STACK_SHARED)
        k_rays<ANY, STATS, PLACE_SHARED><<<blocks, 128, 0, s>>>(S, r, n, (float4*)hits, counters);
    else if (place == PHX_STACK_REGISTER)
        k_rays<ANY, STATS, PLACE_REG_BASE + 1><<<blocks, 128, 0, s>>>(S, r, n, (float4*)hits, counters);
    else
        k_rays<ANY, STATS, PLACE_LOCAL><<<blocks, 128, 0, s>>>(S, r, n, (float4*)hits, counters);
}

}  // namespace
}  // namespace phx

using namespace phx;

// A scene of meshes placed by instances (phx_tracer_create_instanced): each
// mesh's own LBVH over its faces in its own space, the top tree over the
// placed instances' world boxes, the instance records and the emitter
// table's instance column. Absent: one identity instance over tr->bvh.
struct Forest {
    std::vector<phx_mesh> meshes;
    std::vector<std::unique_ptr<BvhWork>> trees;  // per mesh; null for a mesh with no faces
    std::vector<uint32_t> node_base;              // per mesh: its first record in tnodes
    std::vector<phx_instance> insts;              // as given (host)
    std::vector<uint32_t> placed;                 // instances whose mesh has faces
    uint32_t top_records = 1;                     // records kept for the top tree
    uint32_t lamp_cap = 0;                        // entries the emitter table can hold
    BvhWork top;
    DevMem rec, flags, mesh_of, placed_dev, mesh_rec, slots, order_all, lamp_inst, slot_mesh, mesh_off, mesh_list;
};

struct phx_tracer_s {
    Ctx* ctx = nullptr;
    uint32_t nverts = 0, nfaces = 0, nmats = 0, leaf = 4;
    std::unique_ptr<Forest> forest;
    // The tree the walk reads: the LBVH (tr->bvh's Karras array) or the
    // binned SAH tree (sah.rs; its compact array in tr->bvh.nodes/order).
    uint32_t tree = PHX_TREE_LBVH;
    uint32_t sah_count = 0, sah_depth = 0;  // the SAH tree's nodes and depth
    DevMem sah_alt;                          // its refit's second node array
    // The wavefront render's path slots, rays, hits and queues.
    DevMem wf_words, wf_rays, wf_hits, wf_hinst, wf_queues, wf_lens;
    uint32_t* wf_host_lens = nullptr;  // pinned: the queue lengths the host polls
    bool has_normals = false;
    bool emissive = false;  // some material emits: the emitter table is built
    DevMem verts, vnorm, faces, mats, tnodes, tris, tnorm, lamp_slot, lamp_power, lamp_cdf, info, px, rays, cam;
    BvhWork bvh;
    uint32_t w = 0, h = 0;
    uint32_t frame = 0, target = 32;  // Tracer::SAMPLE_COUNT (src/trace/mod.rs:129) until set_samples
    uint32_t kernel = PHX_KERNEL_MEGAKERNEL;  // which render kernel traces a frame (the fastest measured)
    DevMem next;                                 // the state-machine kernel's pixel counter
    uint32_t stack_place = PHX_STACK_LOCAL;      // where thread-per-ray walks keep their stack
    uint32_t walk = PHX_WALK_THREAD;             // ray walks: a thread per ray, persistent warps, sorted first
    DevMem rkeys, rsorted, rorder, ralt_k, ralt_v, rzero;  // the sorted walk's keys and radix-sort scratch
    // The 4-wide tree of PHX_WALK_WIDE, collapsed from the binary tree when
    // first walked after tree_gen moved (every build, refit or tree switch).
    DevMem wide, wide_jobs_a, wide_jobs_b, wide_counts;
    uint32_t tree_gen = 0, wide_gen = 0xFFFFFFFFu, wide_nodes = 0, wide_levels = 0;
    bool have_last = false;
    // Adaptive Sampling, [threshold, min samples, step, on] (Tracer::adapt,
    // set_adaptive): every frame this tracer traces takes it in place of the
    // camera's own (sample.rs:119, `cam.adapt = self.adapt`).
    float adapt[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    phx_camera last;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int32_t prepare_nodes(phx_tracer tr);

int32_t prepare(phx_tracer tr) {
    // After a build or refit: face boxes are in tr->bvh; gather, mark leaf
    // ends, then the walk's nodes, root info and emitter table.
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    const uint32_t n = tr->nfaces;
    const BvhWork& w = tr->bvh;
    k_gather<<<(n + 255) / 256, 256, 0, s>>>((const uint32_t*)w.order.ptr, (const uint4*)tr->faces.ptr,
                                             (const float4*)tr->verts.ptr,
                                             tr->has_normals ? (const float4*)tr->vnorm.ptr : nullptr,
                                             (const float4*)tr->mats.ptr, tr->nmats, n, (float4*)tr->tris.ptr,
                                             tr->has_normals ? (float4*)tr->tnorm.ptr : nullptr, c->status);
    k_mark_ends<<<(n + 255) / 256, 256, 0, s>>>((const float4*)w.nodes.ptr, (const uint32_t*)w.starts.ptr,
                                                w.nstarts(), (float4*)tr->tris.ptr);
    return prepare_nodes(tr);
}

// The LBVH's bounds by k_refit_gather (triangles gathered on the way), after
// enqueue_build(..., refit = false) or on its own for a refit; then the
// walk's nodes as prepare.
int32_t refit_gather(phx_tracer tr) {
    Ctx* c = tr->ctx;
    const uint32_t n = tr->nfaces;
    BvhWork& w = tr->bvh;
    if (n > 0) {
        k_refit_gather<<<(n + 255) / 256, 256, 0, c->stream>>>(
            (const uint32_t*)w.order.ptr, (const uint4*)tr->faces.ptr, (const float4*)tr->verts.ptr,
            tr->has_normals ? (const float4*)tr->vnorm.ptr : nullptr, (const float4*)tr->mats.ptr, tr->nmats,
            (float4*)tr->tris.ptr, tr->has_normals ? (float4*)tr->tnorm.ptr : nullptr, (const uint32_t*)w.parent.ptr,
            (float4*)w.nodes.ptr, (const uint32_t*)w.starts.ptr, w.nstarts(), (uint32_t*)w.counters.ptr, c->status);
        PHX_CUDA(cudaGetLastError());
    }
    return prepare_nodes(tr);
}

// The walk's inner-node records, root info and emitter table from tr->bvh
// and the gathered triangles.
int32_t prepare_nodes(phx_tracer tr) {
    tr->tree_gen++;
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    const uint32_t n = tr->nfaces;
    const BvhWork& w = tr->bvh;
    if (n > 1)
        k_convert<<<(n - 1 + 255) / 256, 256, 0, s>>>((const float4*)w.nodes.ptr, n - 1, (float4*)tr->tnodes.ptr, 0u,
                                                      0u, 0u);
    k_root<<<1, 1, 0, s>>>((const float4*)w.nodes.ptr, n, (float4*)tr->info.ptr, 0u);
    if (tr->emissive)
        k_lamps<<<1, 1024, 0, s>>>((const float4*)tr->tris.ptr, (const float4*)tr->mats.ptr, n,
                                   (uint32_t*)tr->lamp_slot.ptr, (float*)tr->lamp_power.ptr, (float*)tr->lamp_cdf.ptr,
                                   (float4*)tr->info.ptr);
    else  // no material emits: an empty table (the count word of info[2])
        PHX_CUDA(cudaMemsetAsync((float4*)tr->info.ptr + 2, 0, sizeof(float4), s));
    return cuda_check(cudaGetLastError(), "tracer prepare");
}

// A float with the given bits, on the host.
inline float host_bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Instance::inverse and words (instance.rs:60-157) on the host: rows of the
// world matrix (m[col][row] -> row r = m[0..3][r]) and of its inverse (the
// upper 3 x 3 inverted, the translation undone; zero for a singular matrix),
// and the flags (bit 0 at the identity, 1 casts no shadow, 2 mirrors).
void inst_words(const phx_instance& src, float4 out[6], uint32_t* flags) {
    const float* m = src.world;
    auto a = [&](int r, int c) { return m[4 * c + r]; };
    float row[3][4], inv4[3][4];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) row[r][c] = m[4 * c + r];
    const float det = a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
                      a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
    if (std::fabs(det) < 1e-20f) {
        std::memset(inv4, 0, sizeof inv4);
    } else {
        const float d = 1.0f / det;
        const float inv[3][3] = {
            {(a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * d, (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * d,
             (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * d},
            {(a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * d, (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * d,
             (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * d},
            {(a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * d, (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * d,
             (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * d},
        };
        const float t[3] = {m[12], m[13], m[14]};
        for (int r = 0; r < 3; r++) {
            for (int c = 0; c < 3; c++) inv4[r][c] = inv[r][c];
            inv4[r][3] = -((inv[r][0] * t[0] + inv[r][1] * t[1]) + inv[r][2] * t[2]);
        }
    }
    bool identity = true;
    for (int k = 0; k < 16; k++) identity = identity && m[k] == ((k % 5 == 0) ? 1.0f : 0.0f);
    for (int r = 0; r < 3; r++) {
        out[r] = make_float4(row[r][0], row[r][1], row[r][2], row[r][3]);
        out[3 + r] = make_float4(inv4[r][0], inv4[r][1], inv4[r][2], inv4[r][3]);
    }
    *flags = (identity ? 1u : 0u) | (src.casts_shadow ? 0u : 2u) | (det < 0.0f ? 4u : 0u);
}

// The instances' matrices and flags to the device, then Forest::retlas
// (forest.rs:107-121): the top tree over the placed instances' world boxes
// (one instance a leaf), its records, slot table and root info.
int32_t retlas(phx_tracer tr) {
    Forest& F = *tr->forest;
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    const uint32_t ni = (uint32_t)F.insts.size();
    std::vector<float4> rec(8 * (size_t)ni, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    std::vector<uint32_t> flags(ni);
    for (uint32_t i = 0; i < ni; i++) inst_words(F.insts[i], &rec[8 * (size_t)i], &flags[i]);
    // the rows go up (words 6 and 7, the mesh root, are filled on the device)
    for (uint32_t i = 0; i < ni; i++)
        PHX_CUDA(cudaMemcpyAsync((float4*)F.rec.ptr + 8 * (size_t)i, &rec[8 * (size_t)i], 6 * sizeof(float4),
                                 cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(F.flags.ptr, flags.data(), 4 * (size_t)ni, cudaMemcpyHostToDevice, s));
    PHX_TRY(wait_stream(s, 0));  // the host staging vectors go out of scope
    k_inst_fill<<<ceil_div(ni, 128), 128, 0, s>>>((float4*)F.rec.ptr, (const float4*)F.mesh_rec.ptr,
                                                  (const uint32_t*)F.mesh_of.ptr, (const uint32_t*)F.flags.ptr, ni);
    const uint32_t np = (uint32_t)F.placed.size();
    if (np == 0) {  // nothing placed: an empty world (every ray misses)
        const float4 empty[2] = {make_float4(1.0f, 1.0f, 1.0f, host_bits(LEAF | INST)),
                                 make_float4(-1.0f, -1.0f, -1.0f, 1e-3f)};
        PHX_CUDA(cudaMemcpyAsync(tr->info.ptr, empty, sizeof empty, cudaMemcpyHostToDevice, s));
        return cuda_check(cudaGetLastError(), "retlas");
    }
    k_inst_boxes<<<ceil_div(np, 128), 128, 0, s>>>((const float4*)F.rec.ptr, (const uint32_t*)F.placed_dev.ptr, np,
                                                   (phx_aabb*)F.top.prims.ptr);
    PHX_TRY(enqueue_build(c, F.top, np, 1));
    k_inst_slots<<<ceil_div(np, 256), 256, 0, s>>>((const uint32_t*)F.top.order.ptr, (const uint32_t*)F.placed_dev.ptr,
                                                   np, (uint32_t*)F.slots.ptr);
    k_inst_ends<<<ceil_div(np, 256), 256, 0, s>>>((const float4*)F.top.nodes.ptr, (const uint32_t*)F.top.starts.ptr,
                                                  F.top.nstarts(), (uint32_t*)F.slots.ptr);
    if (np > 1)
        k_convert<<<ceil_div(np - 1, 256), 256, 0, s>>>((const float4*)F.top.nodes.ptr, np - 1, (float4*)tr->tnodes.ptr,
                                                        0u, 0u, INST);
    k_root<<<1, 1, 0, s>>>((const float4*)F.top.nodes.ptr, np, (float4*)tr->info.ptr, INST);
    return cuda_check(cudaGetLastError(), "retlas");
}

// A forest's scene preparation after its meshes' trees were built or
// refitted (their face boxes in each tree's prims): slot order, gathered
// triangles, leaf ends, walk records, mesh roots, the top tree, the
// emitter table.
int32_t prepare_forest(phx_tracer tr) {
    Forest& F = *tr->forest;
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    const uint32_t nm = (uint32_t)F.meshes.size();
    for (uint32_t k = 0; k < nm; k++) {
        const BvhWork* w = F.trees[k].get();
        if (!w) continue;
        const uint32_t lo = F.meshes[k].face_lo, n = F.meshes[k].face_hi - lo;
        k_mesh_order<<<ceil_div(n, 256), 256, 0, s>>>((const uint32_t*)w->order.ptr, n, lo,
                                                      (uint32_t*)F.order_all.ptr);
    }
    k_gather<<<ceil_div(tr->nfaces, 256), 256, 0, s>>>(
        (const uint32_t*)F.order_all.ptr, (const uint4*)tr->faces.ptr, (const float4*)tr->verts.ptr,
        tr->has_normals ? (const float4*)tr->vnorm.ptr : nullptr, (const float4*)tr->mats.ptr, tr->nmats, tr->nfaces,
        (float4*)tr->tris.ptr, tr->has_normals ? (float4*)tr->tnorm.ptr : nullptr, c->status);
    for (uint32_t k = 0; k < nm; k++) {
        const BvhWork* w = F.trees[k].get();
        if (!w) continue;
        const uint32_t lo = F.meshes[k].face_lo, n = F.meshes[k].face_hi - lo;
        k_mark_ends<<<ceil_div(n, 256), 256, 0, s>>>((const float4*)w->nodes.ptr, (const uint32_t*)w->starts.ptr,
                                                     w->nstarts(), (float4*)tr->tris.ptr + 3 * (size_t)lo);
        if (n > 1)
            k_convert<<<ceil_div(n - 1, 256), 256, 0, s>>>((const float4*)w->nodes.ptr, n - 1, (float4*)tr->tnodes.ptr,
                                                           F.node_base[k], lo, 0u);
        k_mesh_root<<<1, 1, 0, s>>>((const float4*)w->nodes.ptr, (float4*)F.mesh_rec.ptr + 2 * (size_t)k,
                                    F.node_base[k], lo);
    }
    PHX_TRY(retlas(tr));
    if (tr->emissive)
        k_lamps_inst<<<1, 1024, 0, s>>>((const float4*)tr->tris.ptr, (const float4*)tr->mats.ptr,
                                        (const float4*)F.rec.ptr, (const uint32_t*)F.slot_mesh.ptr,
                                        (const uint32_t*)F.mesh_off.ptr, (const uint32_t*)F.mesh_list.ptr, tr->nfaces,
                                        (uint32_t*)tr->lamp_slot.ptr, (uint32_t*)F.lamp_inst.ptr,
                                        (float*)tr->lamp_power.ptr, (float*)tr->lamp_cdf.ptr, (float4*)tr->info.ptr);
    else
        PHX_CUDA(cudaMemsetAsync((float4*)tr->info.ptr + 2, 0, sizeof(float4), s));
    return cuda_check(cudaGetLastError(), "forest prepare");
}

// Face boxes of every face (into tr->bvh.prims), then each mesh's tree over
// its own range: a fresh build (rebuild) or a refit.
int32_t build_forest(phx_tracer tr, bool rebuild) {
    Forest& F = *tr->forest;
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    PHX_TRY(launch_face_boxes(s, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, tr->nfaces,
                              (phx_aabb*)tr->bvh.prims.ptr));
    for (size_t k = 0; k < F.meshes.size(); k++) {
        BvhWork* w = F.trees[k].get();
        if (!w) continue;
        const uint32_t lo = F.meshes[k].face_lo, n = F.meshes[k].face_hi - lo;
        PHX_CUDA(cudaMemcpyAsync(w->prims.ptr, (const phx_aabb*)tr->bvh.prims.ptr + lo, (size_t)n * sizeof(phx_aabb),
                                 cudaMemcpyDeviceToDevice, s));
        if (rebuild) PHX_TRY(enqueue_build(c, *w, n, tr->leaf));
        else PHX_TRY(enqueue_refit(c, *w, n, false));
    }
    return prepare_forest(tr);
}

// The binned SAH tree (sah.rs:85-189, the tree phiray's tracer walks) over
// the face boxes in tr->bvh.prims, into tr->bvh's node and order arrays,
// then the walk's records: every node of the compact array is reachable, so
// records are indexed by node (leaves skipped) and every leaf marks its end.
int32_t build_sah_tree(phx_tracer tr) {
    Ctx* c = tr->ctx;
    const uint32_t n = tr->nfaces;
    BvhWork& w = tr->bvh;
    PHX_TRY(phx_bvh_build_sah((phx_ctx)((char*)c - offsetof(phx_ctx_s, c)), (const phx_aabb*)w.prims.ptr, n,
                              tr->leaf, (phx_node*)w.nodes.ptr, (uint32_t*)w.order.ptr, &tr->sah_count,
                              &tr->sah_depth));
    return PHX_OK;
}

int32_t prepare_sah(phx_tracer tr) {
    tr->tree_gen++;
    Ctx* c = tr->ctx;
    cudaStream_t s = c->stream;
    const uint32_t n = tr->nfaces, m = tr->sah_count;
    const BvhWork& w = tr->bvh;
    k_gather<<<ceil_div(n, 256), 256, 0, s>>>((const uint32_t*)w.order.ptr, (const uint4*)tr->faces.ptr,
                                              (const float4*)tr->verts.ptr,
                                              tr->has_normals ? (const float4*)tr->vnorm.ptr : nullptr,
                                              (const float4*)tr->mats.ptr, tr->nmats, n, (float4*)tr->tris.ptr,
                                              tr->has_normals ? (float4*)tr->tnorm.ptr : nullptr, c->status);
    k_mark_leaf_ends<<<ceil_div(m, 256), 256, 0, s>>>((const float4*)w.nodes.ptr, m, (float4*)tr->tris.ptr);
    k_convert<<<ceil_div(m, 256), 256, 0, s>>>((const float4*)w.nodes.ptr, m, (float4*)tr->tnodes.ptr, 0u, 0u, 0u);
    k_root<<<1, 1, 0, s>>>((const float4*)w.nodes.ptr, n, (float4*)tr->info.ptr, 0u);
    if (tr->emissive)
        k_lamps<<<1, 1024, 0, s>>>((const float4*)tr->tris.ptr, (const float4*)tr->mats.ptr, n,
                                   (uint32_t*)tr->lamp_slot.ptr, (float*)tr->lamp_power.ptr, (float*)tr->lamp_cdf.ptr,
                                   (float4*)tr->info.ptr);
    else
        PHX_CUDA(cudaMemsetAsync((float4*)tr->info.ptr + 2, 0, sizeof(float4), s));
    return cuda_check(cudaGetLastError(), "SAH prepare");
}

// The SAH tree refitted to the face boxes now in tr->bvh.prims: the
// reference's GPU refit (kernel.rs:130-170, record_refit, gpu.rs:77-85):
// depth + 1 Jacobi passes over every node, rounded up to even so the last
// one lands in the node array.
int32_t refit_sah_tree(phx_tracer tr) {
    Ctx* c = tr->ctx;
    BvhWork& w = tr->bvh;
    const uint32_t m = tr->sah_count;
    PHX_TRY(tr->sah_alt.reserve((size_t)m * 32));
    const uint32_t passes = (tr->sah_depth + 1 + 1) & ~1u;
    phx_refit_param p{};
    p.n = m;
    for (uint32_t k = 0; k < passes; k++) {
        void* bufs[4] = {w.prims.ptr, w.order.ptr, (k & 1) ? tr->sah_alt.ptr : w.nodes.ptr,
                         (k & 1) ? w.nodes.ptr : tr->sah_alt.ptr};
        PHX_TRY(launch_refit_step(c->stream, &p, bufs, m));
    }
    return PHX_OK;
}

// The scene record the kernels take (build-dependent fields are read from
// the device info record inside the kernel, so no host sync is needed).
Scene scene_of(phx_tracer tr) {
    Scene S;
    memset(&S, 0, sizeof S);
    S.nodes = (const float4*)tr->tnodes.ptr;
    S.tris = (const float4*)tr->tris.ptr;
    S.tnorm = tr->has_normals ? (const float4*)tr->tnorm.ptr : nullptr;
    S.mats = (const float4*)tr->mats.ptr;
    S.lamp_slot = (const uint32_t*)tr->lamp_slot.ptr;
    S.lamp_cdf = (const float*)tr->lamp_cdf.ptr;
    S.info = (const float4*)tr->info.ptr;
    if (tr->forest) {
        S.insts = (const float4*)tr->forest->rec.ptr;
        S.inst_slots = (const uint32_t*)tr->forest->slots.ptr;
        S.lamp_inst = (const uint32_t*)tr->forest->lamp_inst.ptr;
    }
    S.nslots = tr->nfaces;
    return S;
}

// Refuses Camera settings the device path does not implement.
int32_t check_camera(const phx_camera* c) {
    if (c->envmap != 0 || c->env_cdf != 0) return fail(PHX_ERR_INVALID, "environment images are not supported");
    if (c->aperture > 0.0f) return fail(PHX_ERR_INVALID, "depth of field (aperture > 0) is not supported");
    if (c->film[0] != 0 || c->film[1] != 0) return fail(PHX_ERR_INVALID, "film transparency/world is not supported");
    if (c->depth[0] != 0) return fail(PHX_ERR_INVALID, "Max Bounces rows (depth) are not supported");
    if (c->integrator[0] != 0.0f) return fail(PHX_ERR_INVALID, "pixel filters other than phiray's own are not supported");
    if (c->view[0] != 0.0f) return fail(PHX_ERR_INVALID, "only the Standard view transform is supported");
    if (c->tile[2] != 0 || c->tile[3] != 0) return fail(PHX_ERR_INVALID, "tiles are not supported");
    if (c->count > PHX_MAX_LIGHT) return fail(PHX_ERR_INVALID, "count %u > 64 lights", c->count);
    if (!(c->scale != 0.0f) || !(c->units != 0.0f) || !(c->aspect != 0.0f))
        return fail(PHX_ERR_INVALID, "scale, units and aspect must be non-zero");
    return PHX_OK;
}

Frame frame_of(const phx_camera* c, uint32_t w, uint32_t h, const phx_light* dev_lights) {
    Frame F;
    F.w = w;
    F.h = h;
    F.n = w * h;
    F.frame0 = 0;
    F.spp = 1;
    F.persp = c->persp;
    F.count = c->count;
    F.bounces = c->bounces;
    F.right = mk(c->right[0], c->right[1], c->right[2]);
    F.up = mk(c->up[0], c->up[1], c->up[2]);
    F.back = mk(c->back[0], c->back[1], c->back[2]);
    F.pivot = mk(c->pivot[0], c->pivot[1], c->pivot[2]);
    F.env = mk(c->env[0], c->env[1], c->env[2]);
    F.scale = c->scale;
    F.units = c->units;
    F.aspect = c->aspect;
    F.dist = c->dist;
    F.pan_x = c->pan[0];
    F.pan_y = c->pan[1];
    F.ao = c->ao;  // the kernel fills ao (when 0) and eps from the extent
    F.eps = 0.0f;
    for (int k = 0; k < 4; k++) F.sky[k] = c->sky[k];
    F.limit_d = c->limit[0];
    F.limit_i = c->limit[1];
    F.exposure = c->view[1];
    F.gamma = c->view[2];
    F.lights = dev_lights;
    // sample.rs:119 passes the resolved Adaptive Sampling setting through;
    // adapt.wgsl reads min and step as u32(adapt.y), max(u32(adapt.z), 1).
    F.adapt_on = c->adapt[3] != 0.0f ? 1u : 0u;
    F.adapt_thr = c->adapt[0];
    F.adapt_min = c->adapt[1] > 0.0f ? (uint32_t)c->adapt[1] : 0u;
    F.adapt_step = c->adapt[2] >= 1.0f ? (uint32_t)c->adapt[2] : 1u;
    F.adapt_list = 0u;
    F.grid = c->grid;
    F.grid_color = make_float4(c->grid_color[0], c->grid_color[1], c->grid_color[2], c->grid_color[3]);
    F.grid_hide = c->grid_hide;
    return F;
}

int32_t ensure_image(phx_tracer tr, uint32_t w, uint32_t h) {
    if (w == 0 || h == 0) return fail(PHX_ERR_INVALID, "image %ux%u", w, h);
    const uint64_t n = (uint64_t)w * h;
    if (n * PHX_PX_LEN + 1 > 0xFFFFFFFFull) return fail(PHX_ERR_INVALID, "image %ux%u is too large", w, h);
    if (tr->w == w && tr->h == h && tr->px.ptr) return PHX_OK;
    PHX_TRY(wait_stream(tr->ctx->stream, 0));
    tr->px.release();
    PHX_TRY(tr->px.reserve((n * PHX_PX_LEN + 1) * 4));
    PHX_CUDA(cudaMemsetAsync(tr->px.ptr, 0, (n * PHX_PX_LEN + 1) * 4, tr->ctx->stream));
    tr->w = w;
    tr->h = h;
    tr->have_last = false;
    return PHX_OK;
}

// The wavefront render's buffers for `count` pixels (grown on demand).
int32_t wf_buffers(phx_tracer tr, uint32_t count, WfBuffers& B) {
    const uint32_t nslots = std::max<uint32_t>(1u, std::min<uint32_t>(count, WF_SLOTS));
    PHX_TRY(tr->wf_words.reserve((size_t)nslots * wf_slot_words() * 4));
    PHX_TRY(tr->wf_rays.reserve((size_t)nslots * 32));
    PHX_TRY(tr->wf_hits.reserve((size_t)nslots * 16));
    PHX_TRY(tr->wf_hinst.reserve((size_t)nslots * 4));
    PHX_TRY(tr->wf_queues.reserve((size_t)3 * nslots * 4));
    PHX_TRY(tr->wf_lens.reserve(16));
    if (!tr->wf_host_lens) PHX_CUDA(cudaHostAlloc((void**)&tr->wf_host_lens, 16, cudaHostAllocDefault));
    B = WfBuffers{nslots,
                  (uint32_t*)tr->wf_words.ptr,
                  (float4*)tr->wf_rays.ptr,
                  (float4*)tr->wf_hits.ptr,
                  (uint32_t*)tr->wf_hinst.ptr,
                  (uint32_t*)tr->wf_queues.ptr,
                  (uint32_t*)tr->wf_lens.ptr,
                  tr->wf_host_lens};
    return PHX_OK;
}

// Launches the tracer's render kernel over pixels [first_px, first_px +
// count_px) of frame F, whose camera is already in tr->cam (no host copy:
// the launch can be recorded into a graph).
// The wide tree of the binary tree the tracer walks now (collapsed on the
// device when the tree changed since the last collapse; waits).
int32_t ensure_wide(phx_tracer tr) {
    if (tr->wide_gen == tr->tree_gen) return PHX_OK;
    Ctx* c = tr->ctx;
    float4 root{};
    PHX_CUDA(cudaMemcpyAsync(&root, tr->info.ptr, sizeof root, cudaMemcpyDeviceToHost, c->stream));
    PHX_TRY(wait_stream(c->stream, 0));
    uint32_t root_ref = 0;
    std::memcpy(&root_ref, &root.w, 4);
    const bool leaf_root = (root_ref & LEAF) != 0;
    const uint32_t ninner = (leaf_root || tr->nfaces < 2) ? 0u : tr->nfaces - 1;
    if (ninner) {
        PHX_TRY(tr->wide.reserve((size_t)ninner * 128));
        PHX_TRY(tr->wide_jobs_a.reserve((size_t)ninner * 8));
        PHX_TRY(tr->wide_jobs_b.reserve((size_t)ninner * 8));
        PHX_TRY(tr->wide_counts.reserve(8));
    }
    PHX_TRY(build_wide((const float4*)tr->tnodes.ptr, ninner, (float4*)tr->wide.ptr, (uint2*)tr->wide_jobs_a.ptr,
                       (uint2*)tr->wide_jobs_b.ptr, (uint32_t*)tr->wide_counts.ptr, c->stream, &tr->wide_nodes,
                       &tr->wide_levels));
    tr->wide_gen = tr->tree_gen;
    return read_status(c);
}

int32_t launch_frame(phx_tracer tr, const Frame& F, f3 sun, uint32_t first_px, uint32_t count_px, bool stats) {
    Ctx* c = tr->ctx;
    uint32_t kernel = tr->kernel;
    const Scene S = scene_of(tr);
    // Adaptive Sampling runs on the megakernel forms (the state machine
    // fetches pixels by index, not from the open list); they all compute
    // the same image, so an adaptive frame takes the default form instead.
    if (F.adapt_on && kernel >= PHX_KERNEL_STATE_MACHINE && kernel <= PHX_KERNEL_STATE_MACHINE_8)
        kernel = PHX_KERNEL_MEGAKERNEL;
    const RenderLaunch L{S,        F,       sun,    (uint32_t*)tr->px.ptr, first_px, count_px,
                         (unsigned long long*)tr->rays.ptr, (uint32_t*)tr->next.ptr, c->sms, c->stream};
    const bool full = tr->forest || F.grid > 0.0f;
    if (kernel == PHX_KERNEL_WAVEFRONT) {
        // the host polls its queues between passes: not while a graph is recorded
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        PHX_CUDA(cudaStreamIsCapturing(c->stream, &cap));
        if (cap != cudaStreamCaptureStatusNone || F.adapt_on) {
            kernel = PHX_KERNEL_MEGAKERNEL;
        } else {
            WfBuffers B;
            PHX_TRY(wf_buffers(tr, count_px, B));
            return render_wavefront(full, stats, L, B);
        }
    }
    if (full) return render_full(kernel, stats, L);
    if (kernel >= PHX_KERNEL_STATE_MACHINE && kernel <= PHX_KERNEL_STATE_MACHINE_8) return render_flat_sm(kernel, stats, L);
    if (kernel >= PHX_KERNEL_MEGAKERNEL_6 && kernel <= PHX_KERNEL_MEGAKERNEL_8_SYNC) return render_flat_b(kernel, stats, L);
    if (kernel >= PHX_KERNEL_MEGAKERNEL_10_SYNC && kernel <= PHX_KERNEL_MEGAKERNEL_16_SYNC)
        return render_flat_c(kernel, stats, L);
    if (kernel >= PHX_KERNEL_MEGAKERNEL_REG && kernel <= PHX_KERNEL_MEGAKERNEL_16_SYNC_REG)
        return render_flat_r(kernel, stats, L);
    return render_flat_a(kernel, stats, L);
}

// The frame record of `cam` for tr, whose lights the kernels read from tr->cam.
Frame frame_for(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first_frame, uint32_t spp) {
    Frame F = frame_of(cam, w, h, ((const phx_camera*)tr->cam.ptr)->lights);
    F.frame0 = first_frame;
    F.spp = spp;
    return F;
}

// Adaptive Sampling's tail after a sample (sample.rs `BTail::Adapt`):
// the convergence check when `sample` is a step boundary past the minimum
// (adapt.wgsl's need_filter), then the dilation and the open-pixel list.
bool adapt_boundary(const Frame& F, uint32_t sample) {
    return sample > F.adapt_min && (sample & (F.adapt_step - 1u)) == F.adapt_step - 1u;
}

int32_t adapt_tail(phx_tracer tr, const Frame& F, bool check, uint32_t sample) {
    cudaStream_t s = tr->ctx->stream;
    uint32_t* px = (uint32_t*)tr->px.ptr;
    const uint32_t blocks = (F.n + 255) / 256;
    if (check && adapt_boundary(F, sample)) k_adapt_check<<<blocks, 256, 0, s>>>(px, F.n, F.adapt_thr);
    k_adapt_dilate<<<blocks, 256, 0, s>>>(px, F.w, F.h);
    PHX_CUDA(cudaMemsetAsync(px + 34ull * F.n, 0, 4, s));
    k_adapt_gather<<<blocks, 256, 0, s>>>(px, F.w, F.h);
    return cuda_check(cudaGetLastError(), "adaptive sampling tail");
}

int32_t launch_render(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first_frame, uint32_t spp,
                      uint32_t first_px, uint32_t count_px, bool stats = false) {
    phx_camera view = *cam;
    std::memcpy(view.adapt, tr->adapt, sizeof view.adapt);
    cam = &view;
    // pageable source: the copy is staged before the call returns
    PHX_CUDA(cudaMemcpyAsync(tr->cam.ptr, cam, sizeof(phx_camera), cudaMemcpyHostToDevice, tr->ctx->stream));
    const Frame F = frame_for(tr, cam, w, h, first_frame, spp);
    const f3 sun = mk(cam->sun[0], cam->sun[1], cam->sun[2]);
    if (!F.adapt_on) return launch_frame(tr, F, sun, first_px, count_px, stats);
    if (first_px != 0 || count_px != F.n)
        return fail(PHX_ERR_INVALID, "adaptive sampling traces whole frames (no pixel slices)");
    // The samples run in launches that end at step boundaries: between two
    // boundaries no pixel's flag changes, so every sample of a launch traces
    // the same open pixels (the reference re-gathers after every sample and
    // gets the same list). Past frame 0 a launch starts from the open list,
    // which is rebuilt first from the flags as they stand.
    uint32_t f = first_frame;
    const uint32_t end = first_frame + spp;
    if (f > 0) PHX_TRY(adapt_tail(tr, F, false, 0));
    while (f < end) {
        uint32_t e = f;
        while (e + 1 < end && !adapt_boundary(F, e)) e++;
        Frame G = F;
        G.frame0 = f;
        G.spp = e - f + 1;
        G.adapt_list = f > 0 ? 1u : 0u;
        PHX_TRY(launch_frame(tr, G, sun, 0, F.n, stats));
        PHX_TRY(adapt_tail(tr, F, true, e));
        f = e + 1;
    }
    return PHX_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// Tracer::new (single identity instance: meshes null) or a scene of meshes
// placed by instances (forest.rs Forest::build).
int32_t create_tracer(phx_ctx ctx, const phx_scene* sc, const phx_mesh* meshes, uint32_t nmeshes,
                      const phx_instance* insts, uint32_t ninsts, phx_tracer* out) {
    if (!ctx || !sc || !out) return fail(PHX_ERR_INVALID, "null argument");
    if (meshes) {
        // Forest::build's assumptions: meshes name ascending, disjoint face
        // ranges; instances name meshes.
        if (nmeshes == 0 || ninsts == 0 || !insts) return fail(PHX_ERR_INVALID, "an instanced scene needs meshes and instances");
        uint32_t at = 0;
        for (uint32_t k = 0; k < nmeshes; k++) {
            if (meshes[k].face_lo < at || meshes[k].face_hi < meshes[k].face_lo || meshes[k].face_hi > sc->nfaces)
                return fail(PHX_ERR_INVALID, "mesh %u: faces [%u, %u) out of order or range", k, meshes[k].face_lo,
                            meshes[k].face_hi);
            at = meshes[k].face_hi;
        }
        for (uint32_t i = 0; i < ninsts; i++)
            if (insts[i].mesh >= nmeshes) return fail(PHX_ERR_INVALID, "instance %u names mesh %u", i, insts[i].mesh);
        if (ninsts >= (1u << 30)) return fail(PHX_ERR_INVALID, "too many instances");
    }
    if (sc->nfaces == 0) return fail(PHX_ERR_INVALID, "a tracer needs at least one face (Tracer::new declines an empty scene)");
    if (!sc->verts || !sc->faces || !sc->mats || sc->nmats == 0 || sc->nverts == 0)
        return fail(PHX_ERR_INVALID, "scene arrays missing");
    if (sc->nfaces >= (1u << 30)) return fail(PHX_ERR_INVALID, "too many faces");
    if (sc->nmats >= (1u << 30)) return fail(PHX_ERR_INVALID, "too many materials");
    PHX_TRY(use(&ctx->c));
    auto* tr = new phx_tracer_s();
    tr->ctx = &ctx->c;
    tr->nverts = sc->nverts;
    tr->nfaces = sc->nfaces;
    tr->nmats = sc->nmats;
    tr->leaf = sc->leaf ? sc->leaf : 4;
    tr->has_normals = sc->normals != nullptr;
    ctx->c.live++;
    cudaStream_t s = ctx->c.stream;
    const size_t n = sc->nfaces;
    int32_t rc = PHX_OK;
    auto step = [&](int32_t r) {
        if (rc == PHX_OK) rc = r;
    };
    step(tr->verts.reserve((size_t)sc->nverts * 16));
    if (tr->has_normals) step(tr->vnorm.reserve((size_t)sc->nverts * 16));
    step(tr->faces.reserve(n * 16));
    step(tr->mats.reserve((size_t)sc->nmats * 128));
    step(tr->tnodes.reserve((n > 1 ? n - 1 : 1) * 64));
    step(tr->tris.reserve(n * 48));
    if (tr->has_normals) step(tr->tnorm.reserve(n * 48));
    step(tr->lamp_slot.reserve(n * 4));
    step(tr->lamp_power.reserve(n * 4));
    step(tr->lamp_cdf.reserve(n * 4));
    step(tr->info.reserve(64));
    step(tr->rays.reserve(24));
    step(tr->cam.reserve(sizeof(phx_camera)));
    step(tr->next.reserve(16));
    step(tr->bvh.reserve(sc->nfaces, ctx->c.sms));
    // Upload, then check the arrays on the device before any kernel indexes
    // through them (faces name vertices and materials; materials take no
    // textures, maps or second lobes) and learn whether some material emits.
    if (rc == PHX_OK)
        rc = cuda_check(cudaMemcpyAsync(tr->verts.ptr, sc->verts, (size_t)sc->nverts * 16, cudaMemcpyHostToDevice, s), "upload");
    if (rc == PHX_OK && tr->has_normals)
        rc = cuda_check(cudaMemcpyAsync(tr->vnorm.ptr, sc->normals, (size_t)sc->nverts * 16, cudaMemcpyHostToDevice, s), "upload");
    if (rc == PHX_OK) rc = cuda_check(cudaMemcpyAsync(tr->faces.ptr, sc->faces, n * 16, cudaMemcpyHostToDevice, s), "upload");
    if (rc == PHX_OK)
        rc = cuda_check(cudaMemcpyAsync(tr->mats.ptr, sc->mats, (size_t)sc->nmats * 128, cudaMemcpyHostToDevice, s), "upload");
    if (rc == PHX_OK) {
        const uint32_t init[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u};
        uint32_t found[4] = {0, 0, 0, 0};
        rc = cuda_check(cudaMemcpyAsync(tr->rays.ptr, init, 16, cudaMemcpyHostToDevice, s), "upload");
        const uint32_t items = std::max<uint32_t>(sc->nfaces, sc->nmats);
        if (rc == PHX_OK) {
            k_check_scene<<<(items + 255) / 256, 256, 0, s>>>((const uint4*)tr->faces.ptr, sc->nfaces, sc->nverts,
                                                               (const float*)tr->mats.ptr, sc->nmats,
                                                               (uint32_t*)tr->rays.ptr);
            rc = cuda_check(cudaGetLastError(), "scene check");
        }
        if (rc == PHX_OK) rc = cuda_check(cudaMemcpyAsync(found, tr->rays.ptr, 16, cudaMemcpyDeviceToHost, s), "check");
        if (rc == PHX_OK) rc = wait_stream(s, 0);
        if (rc == PHX_OK && found[0] != 0xFFFFFFFFu)
            rc = fail(PHX_ERR_INVALID, "face %u names a vertex or material out of range", found[0]);
        if (rc == PHX_OK && found[1] != 0xFFFFFFFFu)
            rc = fail(PHX_ERR_INVALID, "material %u uses a texture (not supported)", found[1]);
        if (rc == PHX_OK && found[2] != 0xFFFFFFFFu)
            rc = fail(PHX_ERR_INVALID, "material %u has a second lobe (not supported)", found[2]);
        tr->emissive = found[3] != 0;
    }
    if (meshes && rc == PHX_OK) {
        tr->forest.reset(new Forest());
        Forest& F = *tr->forest;
        F.meshes.assign(meshes, meshes + nmeshes);
        F.insts.assign(insts, insts + ninsts);
        F.trees.resize(nmeshes);
        F.node_base.assign(nmeshes, 0u);
        std::vector<uint32_t> count(nmeshes, 0u), mesh_of(ninsts), slot_mesh(sc->nfaces, NONE);
        for (uint32_t i = 0; i < ninsts; i++) {
            mesh_of[i] = insts[i].mesh;
            count[insts[i].mesh]++;
            if (meshes[insts[i].mesh].face_hi > meshes[insts[i].mesh].face_lo) F.placed.push_back(i);
        }
        std::vector<uint32_t> off(nmeshes + 1, 0u), list(ninsts);
        for (uint32_t k = 0; k < nmeshes; k++) off[k + 1] = off[k] + count[k];
        std::vector<uint32_t> fill(off.begin(), off.end() - 1);
        for (uint32_t i = 0; i < ninsts; i++) list[fill[insts[i].mesh]++] = i;  // instance order within a mesh
        F.top_records = std::max<uint32_t>(ninsts > 1 ? ninsts - 1 : 1, 1u);
        uint32_t records = F.top_records;
        uint64_t lamps = 0;
        for (uint32_t k = 0; k < nmeshes; k++) {
            const uint32_t n = meshes[k].face_hi - meshes[k].face_lo;
            for (uint32_t f = meshes[k].face_lo; f < meshes[k].face_hi; f++) slot_mesh[f] = k;
            lamps += (uint64_t)n * count[k];
            if (n == 0) continue;
            F.node_base[k] = records;
            records += n - 1;
            F.trees[k].reset(new BvhWork());
            step(F.trees[k]->reserve(n, ctx->c.sms));
        }
        if (lamps >= (1u << 30)) step(fail(PHX_ERR_INVALID, "too many emitter entries"));
        F.lamp_cap = (uint32_t)std::max<uint64_t>(lamps, 1);
        step(F.top.reserve(std::max<uint32_t>(ninsts, 1u), ctx->c.sms));
        step(F.rec.reserve((size_t)ninsts * 8 * 16));
        step(F.flags.reserve((size_t)ninsts * 4));
        step(F.mesh_of.reserve((size_t)ninsts * 4));
        step(F.placed_dev.reserve(std::max<size_t>(F.placed.size(), 1) * 4));
        step(F.mesh_rec.reserve((size_t)nmeshes * 32));
        step(F.slots.reserve((size_t)std::max<uint32_t>(ninsts, 1u) * 4));
        step(F.order_all.reserve(n * 4));
        step(F.lamp_inst.reserve((size_t)F.lamp_cap * 4));
        step(F.slot_mesh.reserve(n * 4));
        step(F.mesh_off.reserve((size_t)(nmeshes + 1) * 4));
        step(F.mesh_list.reserve((size_t)std::max<uint32_t>(ninsts, 1u) * 4));
        step(tr->tnodes.reserve((size_t)records * 64));
        if (tr->emissive) {
            step(tr->lamp_slot.reserve((size_t)F.lamp_cap * 4));
            step(tr->lamp_power.reserve((size_t)F.lamp_cap * 4));
            step(tr->lamp_cdf.reserve((size_t)F.lamp_cap * 4));
        }
        // faces outside every mesh are in no tree: their slots keep their
        // own face, never walked
        std::vector<uint32_t> identity(sc->nfaces);
        for (uint32_t f = 0; f < sc->nfaces; f++) identity[f] = f;
        std::vector<float4> mesh_rec(2 * (size_t)nmeshes, make_float4(0.0f, 0.0f, 0.0f, host_bits(NONE)));
        auto up = [&](DevMem& d, const void* src, size_t bytes) {
            if (rc == PHX_OK && bytes)
                rc = cuda_check(cudaMemcpyAsync(d.ptr, src, bytes, cudaMemcpyHostToDevice, s), "upload");
        };
        up(F.mesh_of, mesh_of.data(), mesh_of.size() * 4);
        up(F.placed_dev, F.placed.data(), F.placed.size() * 4);
        up(F.mesh_rec, mesh_rec.data(), mesh_rec.size() * sizeof(float4));
        up(F.order_all, identity.data(), identity.size() * 4);
        up(F.slot_mesh, slot_mesh.data(), slot_mesh.size() * 4);
        up(F.mesh_off, off.data(), off.size() * 4);
        up(F.mesh_list, list.data(), list.size() * 4);
        if (rc == PHX_OK) rc = wait_stream(s, 0);  // staging vectors go out of scope
    }
    if (rc == PHX_OK) rc = cuda_check(cudaEventCreate(&tr->ev0), "event");
    if (rc == PHX_OK) rc = cuda_check(cudaEventCreate(&tr->ev1), "event");
    if (rc == PHX_OK) rc = cuda_check(cudaMemsetAsync(tr->rays.ptr, 0, 24, s), "zero");
    if (rc == PHX_OK)
        rc = launch_face_boxes(s, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, sc->nfaces,
                               (phx_aabb*)tr->bvh.prims.ptr);
    if (tr->forest) {
        if (rc == PHX_OK) rc = build_forest(tr, true);
    } else {
        if (rc == PHX_OK) rc = enqueue_build(&ctx->c, tr->bvh, sc->nfaces, tr->leaf);
        if (rc == PHX_OK) rc = prepare(tr);
    }
    if (rc == PHX_OK) rc = wait_stream(s, 0);
    if (rc == PHX_OK) rc = read_status(&ctx->c);
    if (rc != PHX_OK) {
        phx_tracer_destroy(tr);
        return rc;
    }
    *out = tr;
    return PHX_OK;
}

}  // namespace

extern "C" {

int32_t phx_tracer_create(phx_ctx ctx, const phx_scene* sc, phx_tracer* out) {
    return create_tracer(ctx, sc, nullptr, 0, nullptr, 0, out);
}

int32_t phx_tracer_create_instanced(phx_ctx ctx, const phx_scene* sc, const phx_mesh* meshes, uint32_t nmeshes,
                                    const phx_instance* insts, uint32_t ninsts, phx_tracer* out) {
    if (!meshes) return fail(PHX_ERR_INVALID, "null mesh table");
    return create_tracer(ctx, sc, meshes, nmeshes, insts, ninsts, out);
}

int32_t phx_tracer_set_tree(phx_tracer tr, uint32_t tree) {
    if (!tr || (tree != PHX_TREE_LBVH && tree != PHX_TREE_SAH)) return fail(PHX_ERR_INVALID, "bad argument");
    if (tr->forest && tree != PHX_TREE_LBVH)
        return fail(PHX_ERR_INVALID, "scenes of instances keep LBVH mesh trees");
    PHX_TRY(use(tr->ctx));
    cudaStream_t s = tr->ctx->stream;
    if (tree == PHX_TREE_SAH) PHX_TRY(tr->tnodes.reserve((size_t)(2 * tr->nfaces - 1) * 64));
    PHX_TRY(launch_face_boxes(s, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, tr->nfaces,
                              (phx_aabb*)tr->bvh.prims.ptr));
    tr->tree = tree;
    if (tree == PHX_TREE_SAH) {
        PHX_TRY(build_sah_tree(tr));
        PHX_TRY(prepare_sah(tr));
    } else {
        PHX_TRY(enqueue_build(tr->ctx, tr->bvh, tr->nfaces, tr->leaf));
        PHX_TRY(prepare(tr));
    }
    tr->have_last = false;
    PHX_TRY(wait_stream(s, 0));
    return read_status(tr->ctx);
}

int32_t phx_tracer_autotune_tree(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t spp,
                                 uint32_t frames, uint32_t* chosen, float* ms) {
    if (!tr || !cam || spp == 0) return fail(PHX_ERR_INVALID, "bad argument");
    if (tr->forest) return fail(PHX_ERR_INVALID, "scenes of instances keep LBVH mesh trees");
    PHX_TRY(use(tr->ctx));
    cudaStream_t s = tr->ctx->stream;
    float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    cudaEvent_t a = nullptr, b = nullptr;
    PHX_CUDA(cudaEventCreate(&a));
    PHX_CUDA(cudaEventCreate(&b));
    int32_t rc = PHX_OK;
    for (uint32_t k = 0; k < 2 && rc == PHX_OK; k++) {
        // build (from the face boxes), then a trace of spp samples, each timed
        // after an untimed one (a process's first build of a kind also pays
        // one-time costs: kernel loading, pool growth)
        const uint32_t tree = k == 0 ? PHX_TREE_LBVH : PHX_TREE_SAH;
        rc = phx_tracer_set_tree(tr, tree);
        if (rc == PHX_OK) rc = cuda_check(cudaEventRecord(a, s), "event");
        if (rc == PHX_OK) rc = phx_tracer_set_tree(tr, tree);
        if (rc == PHX_OK) rc = cuda_check(cudaEventRecord(b, s), "event");
        if (rc == PHX_OK) rc = wait_stream(s, 0);
        if (rc == PHX_OK) rc = cuda_check(cudaEventElapsedTime(&t[2 * k], a, b), "event");
        if (rc == PHX_OK) rc = phx_tracer_trace(tr, cam, w, h, 0, spp);  // warms the kernel and the tree
        if (rc == PHX_OK) rc = cuda_check(cudaEventRecord(a, s), "event");
        if (rc == PHX_OK) rc = phx_tracer_trace(tr, cam, w, h, 0, spp);
        if (rc == PHX_OK) rc = cuda_check(cudaEventRecord(b, s), "event");
        if (rc == PHX_OK) rc = wait_stream(s, 0);
        if (rc == PHX_OK) rc = cuda_check(cudaEventElapsedTime(&t[2 * k + 1], a, b), "event");
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    PHX_TRY(rc);
    // build once, then `frames` traces of spp samples each
    const double lbvh = t[0] + (double)frames * t[1], sah = t[2] + (double)frames * t[3];
    const uint32_t pick = sah < lbvh ? PHX_TREE_SAH : PHX_TREE_LBVH;
    if (pick != tr->tree) PHX_TRY(phx_tracer_set_tree(tr, pick));
    if (chosen) *chosen = pick;
    if (ms) std::memcpy(ms, t, sizeof t);
    return PHX_OK;
}

int32_t phx_tracer_reinstance(phx_tracer tr, const phx_instance* insts, uint32_t ninsts) {
    if (!tr || !insts) return fail(PHX_ERR_INVALID, "null argument");
    if (!tr->forest) return fail(PHX_ERR_INVALID, "the tracer was not built with instances");
    Forest& F = *tr->forest;
    if (ninsts != F.insts.size()) return fail(PHX_ERR_INVALID, "instance count %u, the tracer holds %zu", ninsts, F.insts.size());
    for (uint32_t i = 0; i < ninsts; i++)
        if (insts[i].mesh != F.insts[i].mesh) return fail(PHX_ERR_INVALID, "instance %u changed its mesh", i);
    PHX_TRY(use(tr->ctx));
    F.insts.assign(insts, insts + ninsts);
    PHX_TRY(retlas(tr));
    if (tr->emissive)
        k_lamps_inst<<<1, 1024, 0, tr->ctx->stream>>>(
            (const float4*)tr->tris.ptr, (const float4*)tr->mats.ptr, (const float4*)F.rec.ptr,
            (const uint32_t*)F.slot_mesh.ptr, (const uint32_t*)F.mesh_off.ptr, (const uint32_t*)F.mesh_list.ptr,
            tr->nfaces, (uint32_t*)tr->lamp_slot.ptr, (uint32_t*)F.lamp_inst.ptr, (float*)tr->lamp_power.ptr,
            (float*)tr->lamp_cdf.ptr, (float4*)tr->info.ptr);
    tr->have_last = false;  // the image starts again
    return cuda_check(cudaGetLastError(), "reinstance");
}

int32_t phx_tracer_destroy(phx_tracer tr) {
    if (!tr) return PHX_OK;
    use(tr->ctx);
    cudaStreamSynchronize(tr->ctx->stream);
    if (tr->ev0) cudaEventDestroy(tr->ev0);
    if (tr->ev1) cudaEventDestroy(tr->ev1);
    if (tr->wf_host_lens) cudaFreeHost(tr->wf_host_lens);
    tr->ctx->live--;
    delete tr;
    return PHX_OK;
}

int32_t phx_tracer_set_kernel(phx_tracer tr, uint32_t kernel) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (kernel >= PHX_KERNEL_COUNT) return fail(PHX_ERR_INVALID, "unknown render kernel %u", kernel);
    tr->kernel = kernel;
    return PHX_OK;
}

int32_t phx_tracer_autotune(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t spp,
                            uint32_t* chosen, float* ms) {
    if (!tr || !cam) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    PHX_TRY(ensure_image(tr, w, h));
    Ctx* c = tr->ctx;
    float best = 0.0f;
    uint32_t pick = PHX_KERNEL_STATE_MACHINE;
    const uint32_t keep = tr->kernel;
    for (uint32_t k = 0; k < PHX_KERNEL_COUNT; k++) {
        tr->kernel = k;
        PHX_TRY(launch_render(tr, cam, w, h, 0, spp ? spp : 1, 0, w * h));  // warm-up
        PHX_CUDA(cudaEventRecord(tr->ev0, c->stream));
        PHX_TRY(launch_render(tr, cam, w, h, 0, spp ? spp : 1, 0, w * h));
        PHX_CUDA(cudaEventRecord(tr->ev1, c->stream));
        PHX_TRY(wait_stream(c->stream, 60000));
        float t = 0.0f;
        PHX_CUDA(cudaEventElapsedTime(&t, tr->ev0, tr->ev1));
        if (ms) ms[k] = t;
        if (k == 0 || t < best) {
            best = t;
            pick = k;
        }
    }
    tr->kernel = pick;
    (void)keep;
    tr->have_last = false;  // the image holds the tuning frames: start over
    if (chosen) *chosen = pick;
    return read_status(c);
}

int32_t phx_tracer_set_stack(phx_tracer tr, uint32_t place) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (place > PHX_STACK_REGISTER) return fail(PHX_ERR_INVALID, "unknown stack placement %u", place);
    tr->stack_place = place;
    return PHX_OK;
}

int32_t phx_tracer_set_walk(phx_tracer tr, uint32_t mode) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (mode > PHX_WALK_WIDE_THREAD) return fail(PHX_ERR_INVALID, "unknown walk mode %u", mode);
    if (mode >= PHX_WALK_WIDE && tr->forest)
        return fail(PHX_ERR_INVALID, "the wide walk takes single-instance scenes");
    tr->walk = mode;
    return PHX_OK;
}

int32_t phx_tracer_set_samples(phx_tracer tr, uint32_t samples) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    tr->target = samples ? samples : 1;
    return PHX_OK;
}

int32_t phx_tracer_trace(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first, uint32_t spp) {
    if (!tr || !cam) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    PHX_TRY(ensure_image(tr, w, h));
    if (spp == 0) return PHX_OK;
    Ctx* c = tr->ctx;
    PHX_CUDA(cudaMemsetAsync(tr->rays.ptr, 0, 8, c->stream));
    PHX_CUDA(cudaEventRecord(tr->ev0, c->stream));
    PHX_TRY(launch_render(tr, cam, w, h, first, spp, 0, w * h));
    PHX_CUDA(cudaEventRecord(tr->ev1, c->stream));
    tr->frame = first + spp - 1;
    tr->last = *cam;
    std::memcpy(tr->last.adapt, tr->adapt, sizeof tr->adapt);
    tr->have_last = true;
    return PHX_OK;
}

int32_t phx_tracer_trace_rows(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                              uint32_t spp, uint32_t row0, uint32_t rows) {
    if (!tr || !cam) return fail(PHX_ERR_INVALID, "null argument");
    if (row0 > h || rows > h - row0) return fail(PHX_ERR_INVALID, "rows [%u, %u) outside the %u-row frame", row0, row0 + rows, h);
    if (tr->adapt[3] != 0.0f) return fail(PHX_ERR_INVALID, "adaptive sampling traces whole frames");
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    PHX_TRY(ensure_image(tr, w, h));
    if (spp == 0 || rows == 0) return PHX_OK;
    Ctx* c = tr->ctx;
    PHX_CUDA(cudaMemsetAsync(tr->rays.ptr, 0, 8, c->stream));
    PHX_CUDA(cudaEventRecord(tr->ev0, c->stream));
    PHX_TRY(launch_render(tr, cam, w, h, first, spp, row0 * w, rows * w));
    PHX_CUDA(cudaEventRecord(tr->ev1, c->stream));
    tr->frame = first + spp - 1;
    tr->last = *cam;
    std::memcpy(tr->last.adapt, tr->adapt, sizeof tr->adapt);
    tr->have_last = true;
    return PHX_OK;
}

// The planes a traced row carries, as (first plane, words a pixel): packed,
// linear sums, shown, albedo, normal, depth, overlay, coverage, film,
// outline, sample count, missed (read.rs:37-56).
static const uint32_t ROW_PLANES[12][2] = {{0, 1},  {1, 3},  {4, 3},  {7, 3},  {10, 3}, {13, 1},
                                            {20, 3}, {23, 1}, {24, 1}, {25, 1}, {31, 1}, {33, 1}};

int32_t phx_tracer_copy_rows(phx_tracer tr, uint32_t row0, uint32_t rows, uint32_t* packed, int32_t into_image) {
    if (!tr || (rows && !packed)) return fail(PHX_ERR_INVALID, "null argument");
    if (!tr->px.ptr) return fail(PHX_ERR_INVALID, "no image yet");
    if (row0 > tr->h || rows > tr->h - row0) return fail(PHX_ERR_INVALID, "rows outside the frame");
    PHX_TRY(use(tr->ctx));
    const size_t n = (size_t)tr->w * tr->h, w = tr->w;
    uint32_t* px = (uint32_t*)tr->px.ptr;
    size_t at = 0;
    for (const auto& pl : ROW_PLANES) {
        uint32_t* img = px + pl[0] * n + (size_t)pl[1] * row0 * w;
        const size_t words = (size_t)pl[1] * rows * w;
        if (words) {
            if (into_image)
                PHX_CUDA(cudaMemcpyAsync(img, packed + at, words * 4, cudaMemcpyDeviceToDevice, tr->ctx->stream));
            else
                PHX_CUDA(cudaMemcpyAsync(packed + at, img, words * 4, cudaMemcpyDeviceToDevice, tr->ctx->stream));
        }
        at += words;
    }
    return PHX_OK;
}

int32_t phx_tracer_sample(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t slices,
                          const volatile int32_t* cancel, uint32_t* frame, int32_t* done) {
    if (!tr || !cam) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    w = w ? w : 1;
    h = h ? h : 1;
    PHX_TRY(ensure_image(tr, w, h));
    const uint32_t n = w * h;
    slices = slices < 1 ? 1 : (slices > n ? n : slices);
    if (tr->adapt[3] != 0.0f) slices = 1;  // an adaptive sample traces the open list whole
    // sample.rs:119-134: the tracer's Adaptive Sampling setting stamped on
    // the view; the same view (everything past n, groups_x) is the next
    // frame, another view starts over.
    phx_camera view = *cam;
    std::memcpy(view.adapt, tr->adapt, sizeof view.adapt);
    cam = &view;
    const bool same = tr->have_last && memcmp((const char*)&tr->last + 8, (const char*)cam + 8, sizeof(phx_camera) - 8) == 0;
    if (same && tr->frame + 1 >= tr->target) {
        if (frame) *frame = tr->frame;
        if (done) *done = 1;
        return PHX_OK;
    }
    const uint32_t f = same ? tr->frame + 1 : 0;
    Ctx* c = tr->ctx;
    PHX_CUDA(cudaMemsetAsync(tr->rays.ptr, 0, 8, c->stream));
    PHX_CUDA(cudaEventRecord(tr->ev0, c->stream));
    for (uint32_t k = 0; k < slices; k++) {
        const uint32_t a = (uint32_t)((uint64_t)n * k / slices), b = (uint32_t)((uint64_t)n * (k + 1) / slices);
        PHX_TRY(launch_render(tr, cam, w, h, f, 1, a, b - a));
        if (slices > 1) {
            PHX_TRY(wait_stream(c->stream, 0));
            if (cancel && *cancel) {
                tr->have_last = false;  // a half-sampled frame is no frame
                return fail(PHX_ERR_CANCELLED, "sample cancelled after slice %u of %u", k + 1, slices);
            }
        }
    }
    PHX_CUDA(cudaEventRecord(tr->ev1, c->stream));
    tr->frame = f;
    tr->last = *cam;
    tr->have_last = true;
    if (frame) *frame = f;
    if (done) *done = (f + 1 >= tr->target) ? 1 : 0;
    return PHX_OK;
}

int32_t phx_tracer_show(phx_tracer tr, const float* linear, uint64_t count) {
    if (!tr || (!linear && count)) return fail(PHX_ERR_INVALID, "null argument");
    if (!tr->px.ptr || !tr->have_last) return fail(PHX_ERR_INVALID, "no image to show yet");
    PHX_TRY(use(tr->ctx));
    const uint64_t n = (uint64_t)tr->w * tr->h;
    cudaStream_t s = tr->ctx->stream;
    // read.rs:182-216: the sums are k times the mean, k the samples each
    // pixel took (counts: frame + 1, or the pixel's own count under
    // Adaptive Sampling); missing pixels of `linear` read as 0.
    std::vector<uint32_t> cnt;
    if (tr->adapt[3] != 0.0f) {
        cnt.resize(n);
        PHX_CUDA(cudaMemcpyAsync(cnt.data(), (const uint32_t*)tr->px.ptr + 31 * n, n * 4, cudaMemcpyDeviceToHost, s));
        PHX_TRY(wait_stream(s, 0));
    }
    std::vector<float> sums(3 * n, 0.0f);
    for (uint64_t i = 0; i < n; i++) {
        const float k = tr->adapt[3] != 0.0f ? (float)(cnt[i] > 1u ? cnt[i] : 1u) : (float)(tr->frame + 1);
        for (int c = 0; c < 3; c++) sums[3 * i + c] = i < count ? linear[3 * i + c] * k : 0.0f * k;
    }
    PHX_CUDA(cudaMemcpyAsync((uint32_t*)tr->px.ptr + n, sums.data(), 3 * n * 4, cudaMemcpyHostToDevice, s));
    k_show<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((uint32_t*)tr->px.ptr, (uint32_t)n, tr->last.view[1],
                                                       tr->last.view[2]);
    PHX_TRY(cuda_check(cudaGetLastError(), "show"));
    return wait_stream(s, 0);  // `linear` is the caller's: the copy has read it
}

int32_t phx_tracer_set_adaptive(phx_tracer tr, const float adapt[4]) {
    if (!tr || !adapt) return fail(PHX_ERR_INVALID, "null argument");
    if (std::memcmp(tr->adapt, adapt, sizeof tr->adapt) != 0) {
        std::memcpy(tr->adapt, adapt, sizeof tr->adapt);
        tr->have_last = false;  // another setting is another view: the next sample starts over
    }
    return PHX_OK;
}

int32_t phx_tracer_unconverged(phx_tracer tr, uint32_t* count, uint32_t timeout_ms) {
    if (!tr || !count) return fail(PHX_ERR_INVALID, "null argument");
    if (tr->adapt[3] == 0.0f) return fail(PHX_ERR_INVALID, "adaptive sampling is off");
    if (!tr->px.ptr) return fail(PHX_ERR_INVALID, "nothing traced yet");
    PHX_TRY(use(tr->ctx));
    const uint64_t n = (uint64_t)tr->w * tr->h;
    PHX_CUDA(cudaMemcpyAsync(count, (const uint32_t*)tr->px.ptr + 34 * n, 4, cudaMemcpyDeviceToHost, tr->ctx->stream));
    PHX_TRY(wait_stream(tr->ctx->stream, timeout_ms));
    return read_status(tr->ctx);
}

int32_t phx_tracer_read(phx_tracer tr, uint64_t offset, uint32_t* dst, uint64_t count, uint32_t timeout_ms) {
    if (!tr || (!dst && count)) return fail(PHX_ERR_INVALID, "null argument");
    const uint64_t words = (uint64_t)tr->w * tr->h * PHX_PX_LEN + 1;
    if (!tr->px.ptr || offset + count > words) return fail(PHX_ERR_INVALID, "read past the image");
    PHX_TRY(use(tr->ctx));
    PHX_CUDA(cudaMemcpyAsync(dst, (const uint32_t*)tr->px.ptr + offset, count * 4, cudaMemcpyDeviceToHost, tr->ctx->stream));
    PHX_TRY(wait_stream(tr->ctx->stream, timeout_ms));
    return read_status(tr->ctx);
}

int32_t phx_tracer_verts(phx_tracer tr, float** verts, uint32_t* nverts) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (verts) *verts = (float*)tr->verts.ptr;
    if (nverts) *nverts = tr->nverts;
    return PHX_OK;
}

int32_t phx_tracer_image(phx_tracer tr, uint32_t** px, uint64_t* words) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (px) *px = (uint32_t*)tr->px.ptr;
    if (words) *words = tr->px.ptr ? (uint64_t)tr->w * tr->h * PHX_PX_LEN + 1 : 0;
    return PHX_OK;
}

int32_t phx_tracer_denoise(phx_tracer tr, int32_t keep) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    if (!tr->px.ptr || !tr->have_last) return PHX_OK;  // nothing traced: read.rs:90
    PHX_TRY(use(tr->ctx));
    const float strength[4] = {64.0f, 8.0f, 40.0f, 7.0f};
    return phx_denoise((phx_ctx)((char*)tr->ctx - offsetof(phx_ctx_s, c)), (uint32_t*)tr->px.ptr, tr->w, tr->h,
                       strength, tr->last.view, keep);
}

int32_t phx_tracer_snapshot(phx_tracer tr, float* snap) {
    if (!tr || !snap) return fail(PHX_ERR_INVALID, "null argument");
    if (!tr->px.ptr) return fail(PHX_ERR_INVALID, "nothing traced");
    PHX_TRY(use(tr->ctx));
    return phx_nn_snapshot((phx_ctx)((char*)tr->ctx - offsetof(phx_ctx_s, c)), (const uint32_t*)tr->px.ptr, tr->w,
                           tr->h, snap);
}

int32_t phx_tracer_denoise_learned(phx_tracer tr, phx_unet net, const float* half, int32_t tile, float threshold,
                                   int32_t keep, uint32_t* fallback) {
    if (!tr || !net) return fail(PHX_ERR_INVALID, "null argument");
    if (fallback) *fallback = 0;
    if (!tr->px.ptr || !tr->have_last) return PHX_OK;  // nothing traced: read.rs:90
    PHX_TRY(use(tr->ctx));
    return phx_unet_denoise_px(net, (uint32_t*)tr->px.ptr, half, tr->w, tr->h, tr->last.view, tile, threshold, keep,
                               fallback);
}

int32_t phx_tracer_time(phx_tracer tr, float* gpu_ms, uint64_t* rays) {
    if (!tr) return fail(PHX_ERR_INVALID, "null tracer");
    PHX_TRY(use(tr->ctx));
    PHX_TRY(wait_stream(tr->ctx->stream, 0));
    if (gpu_ms) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, tr->ev0, tr->ev1) != cudaSuccess) {
            cudaGetLastError();
            ms = 0.0f;
        }
        *gpu_ms = ms;
    }
    if (rays) PHX_CUDA(cudaMemcpy(rays, tr->rays.ptr, 8, cudaMemcpyDeviceToHost));
    return read_status(tr->ctx);
}

int32_t phx_tracer_repose_device(phx_tracer tr, const float* verts, int32_t rebuild) {
    if (!tr || !verts) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(tr->ctx));
    cudaStream_t s = tr->ctx->stream;
    if ((const void*)verts != tr->verts.ptr)
        PHX_CUDA(cudaMemcpyAsync(tr->verts.ptr, verts, (size_t)tr->nverts * 16, cudaMemcpyDeviceToDevice, s));
    if (tr->forest) {  // Tracer::repose: each mesh's tree refitted (or rebuilt), the top tree again
        PHX_TRY(build_forest(tr, rebuild != 0));
        tr->have_last = false;
        return PHX_OK;
    }
    if (tr->tree == PHX_TREE_SAH) {
        PHX_TRY(launch_face_boxes(s, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, tr->nfaces,
                                  (phx_aabb*)tr->bvh.prims.ptr));
        if (rebuild) PHX_TRY(build_sah_tree(tr));
        else PHX_TRY(refit_sah_tree(tr));
        PHX_TRY(prepare_sah(tr));
        tr->have_last = false;
        return PHX_OK;
    }
    // The LBVH: a rebuild sorts the face boxes; its bounds, like a refit's,
    // come from k_refit_gather, which takes each face's box from the
    // vertices (so a refit leaves tr->bvh.prims as it was: every user of
    // the face boxes computes them first).
    if (rebuild) {
        PHX_TRY(launch_face_boxes(s, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, tr->nfaces,
                                  (phx_aabb*)tr->bvh.prims.ptr));
        PHX_TRY(enqueue_build(tr->ctx, tr->bvh, tr->nfaces, tr->leaf, Gate{}, false));
    }
    PHX_TRY(refit_gather(tr));
    tr->have_last = false;  // a new pose starts the image over
    return PHX_OK;
}

int32_t phx_tracer_primary(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t frame, uint32_t* ids,
                           float* ts) {
    if (!tr || !cam || !ids || !ts) return fail(PHX_ERR_INVALID, "null argument");
    if (w == 0 || h == 0) return fail(PHX_ERR_INVALID, "image %ux%u", w, h);
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    const Scene S = scene_of(tr);
    const Frame F = frame_of(cam, w, h, nullptr);
    k_primary<<<(w * h + 127) / 128, 128, 0, tr->ctx->stream>>>(S, F, frame, ids, ts);
    return cuda_check(cudaGetLastError(), "primary");
}

int32_t phx_tracer_secondary_rays(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t frame,
                                  float* rays) {
    if (!tr || !cam || !rays) return fail(PHX_ERR_INVALID, "null argument");
    if (w == 0 || h == 0) return fail(PHX_ERR_INVALID, "image %ux%u", w, h);
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    const Scene S = scene_of(tr);
    const Frame F = frame_of(cam, w, h, nullptr);
    k_secondary<<<(w * h + 127) / 128, 128, 0, tr->ctx->stream>>>(S, F, frame, (float4*)rays);
    return cuda_check(cudaGetLastError(), "secondary rays");
}

namespace phx {
namespace {
// Sorts the rays' keys (k_ray_keys) with the stable radix sort: the order
// the sorted walk takes them in. Stream-ordered.
int32_t sort_rays(phx_tracer tr, const Scene& S, const float* rays, uint32_t n, const uint32_t** order) {
    Ctx* c = tr->ctx;
    const uint32_t stride = (n + 4095) / 4096;
    const size_t zero_words = 4 * 256 + 16 + (size_t)4 * stride * 256;
    PHX_TRY(tr->rkeys.reserve((size_t)n * 4));
    PHX_TRY(tr->rsorted.reserve((size_t)n * 4));
    PHX_TRY(tr->rorder.reserve((size_t)n * 4));
    PHX_TRY(tr->ralt_k.reserve((size_t)n * 4));
    PHX_TRY(tr->ralt_v.reserve((size_t)n * 4));
    PHX_TRY(tr->rzero.reserve(zero_words * 4));
    PHX_CUDA(cudaMemsetAsync(tr->rzero.ptr, 0, zero_words * 4, c->stream));
    k_ray_keys<<<(n + 255) / 256, 256, 0, c->stream>>>(S, (const float4*)rays, n, (uint32_t*)tr->rkeys.ptr);
    PHX_CUDA(cudaGetLastError());
    uint32_t* z = (uint32_t*)tr->rzero.ptr;
    PHX_TRY(enqueue_sort_raw(c, (const uint32_t*)tr->rkeys.ptr, n, (uint32_t*)tr->rorder.ptr,
                             (uint32_t*)tr->rsorted.ptr, (uint32_t*)tr->ralt_k.ptr, (uint32_t*)tr->ralt_v.ptr, z,
                             z + 4 * 256, z + 4 * 256 + 16, stride));
    *order = (const uint32_t*)tr->rorder.ptr;
    return PHX_OK;
}
}  // namespace
}  // namespace phx


int32_t phx_trace_rays(phx_tracer tr, const float* rays, uint32_t n, float* hits, int32_t any_hit) {
    if (!tr || (n && (!rays || !hits))) return fail(PHX_ERR_INVALID, "null argument");
    if (n == 0) return PHX_OK;
    PHX_TRY(use(tr->ctx));
    const Scene S = scene_of(tr);
    if (tr->walk >= PHX_WALK_WIDE) {
        PHX_TRY(ensure_wide(tr));
        return launch_rays_wide(S, (const float4*)tr->wide.ptr, rays, n, hits, any_hit != 0, nullptr,
                                tr->walk == PHX_WALK_WIDE ? (uint32_t*)tr->next.ptr : nullptr, tr->ctx->sms,
                                tr->ctx->stream);
    }
    uint32_t* nx = tr->walk != PHX_WALK_THREAD ? (uint32_t*)tr->next.ptr : nullptr;
    const uint32_t* order = nullptr;
    if (tr->walk == PHX_WALK_SORTED) PHX_TRY(sort_rays(tr, S, rays, n, &order));
    if (any_hit)
        launch_rays<true, false>(S, rays, n, hits, nullptr, tr->stack_place, tr->ctx->stream, nx, tr->ctx->sms, order);
    else
        launch_rays<false, false>(S, rays, n, hits, nullptr, tr->stack_place, tr->ctx->stream, nx, tr->ctx->sms, order);
    return cuda_check(cudaGetLastError(), "trace rays");
}

int32_t phx_trace_rays_stats(phx_tracer tr, const float* rays, uint32_t n, float* hits, int32_t any_hit,
                             uint64_t counts[3]) {
    if (!tr || !counts || (n && (!rays || !hits))) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(tr->ctx));
    cudaStream_t s = tr->ctx->stream;
    PHX_CUDA(cudaMemsetAsync(tr->rays.ptr, 0, 24, s));
    const Scene S = scene_of(tr);
    if (n && tr->walk >= PHX_WALK_WIDE) {
        PHX_TRY(ensure_wide(tr));
        PHX_TRY(launch_rays_wide(S, (const float4*)tr->wide.ptr, rays, n, hits, any_hit != 0,
                                 (unsigned long long*)tr->rays.ptr,
                                 tr->walk == PHX_WALK_WIDE ? (uint32_t*)tr->next.ptr : nullptr, tr->ctx->sms, s));
    } else if (n) {
        uint32_t* nx = tr->walk != PHX_WALK_THREAD ? (uint32_t*)tr->next.ptr : nullptr;
        const uint32_t* order = nullptr;
        if (tr->walk == PHX_WALK_SORTED) PHX_TRY(sort_rays(tr, S, rays, n, &order));
        unsigned long long* ct = (unsigned long long*)tr->rays.ptr;
        if (any_hit) launch_rays<true, true>(S, rays, n, hits, ct, tr->stack_place, s, nx, tr->ctx->sms, order);
        else launch_rays<false, true>(S, rays, n, hits, ct, tr->stack_place, s, nx, tr->ctx->sms, order);
        PHX_CUDA(cudaGetLastError());
    }
    PHX_CUDA(cudaMemcpyAsync(counts, tr->rays.ptr, 24, cudaMemcpyDeviceToHost, s));
    PHX_TRY(wait_stream(s, 0));
    counts[0] = n;
    return PHX_OK;
}

int32_t phx_tracer_trace_stats(phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                               uint32_t spp, uint64_t counts[3]) {
    if (!tr || !cam || !counts) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(check_camera(cam));
    PHX_TRY(use(tr->ctx));
    PHX_TRY(ensure_image(tr, w, h));
    cudaStream_t s = tr->ctx->stream;
    PHX_CUDA(cudaMemsetAsync(tr->rays.ptr, 0, 24, s));
    if (spp) PHX_TRY(launch_render(tr, cam, w, h, first, spp, 0, w * h, true));
    PHX_CUDA(cudaMemcpyAsync(counts, tr->rays.ptr, 24, cudaMemcpyDeviceToHost, s));
    PHX_TRY(wait_stream(s, 0));
    tr->frame = first + spp - 1;
    tr->last = *cam;
    std::memcpy(tr->last.adapt, tr->adapt, sizeof tr->adapt);
    tr->have_last = true;
    return read_status(tr->ctx);
}

}  // extern "C"

// ---- batched serving: many tracers' frames in one persistent launch ----

namespace phx {
namespace {

// A serving frame of many scenes can take seconds: the batch's host waits
// allow two minutes before they report PHX_ERR_TIMEOUT.
constexpr uint32_t BATCH_WAIT_MS = 120000;

__global__ void k_stamp(unsigned long long* dst) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    *dst = t;
}

struct BatchJob {
    phx_tracer tr;
    phx_camera cam;
    uint32_t w, h, first, spp;
};

}  // namespace
}  // namespace phx

struct phx_batch_s {
    phx_ctx handle = nullptr;
    Ctx* ctx = nullptr;
    std::vector<BatchJob> jobs;
    std::vector<uint32_t> order;  // jobs by decreasing per-tile cost
    uint32_t kind = PHX_BATCH_PERSISTENT, threads = 128, stack = PHX_STACK_LOCAL;
    DevMem djobs, next, counters, stamps, modes;
    uint32_t* host_modes = nullptr;  // pinned: the graph's per-replay copy source
    uint32_t ntiles = 0;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<phx_unet> nets;  // one network per padded image shape
    std::vector<int> net_of;     // job -> nets index (-1: the a-trous Denoise)
};

namespace phx {
namespace {

// The batch kernel in full mode when some job's scene is one of instances or
// its frame draws the floor grid (that mode takes every job).
template <int THREADS>
int32_t launch_batch(phx_batch b) {
    bool full = false;
    for (const BatchJob& bj : b->jobs) full = full || bj.tr->forest || bj.cam.grid > 0.0f;
    Ctx* c = b->ctx;
    return render_batch(THREADS, full, b->stack == PHX_STACK_SHARED, b->kind == PHX_BATCH_PERSISTENT_DENSE, c->device,
                        c->sms, b->djobs.ptr, (uint32_t)b->jobs.size(), b->ntiles, (uint32_t*)b->next.ptr, c->stream);
}

// Uploads cameras and the job table (host copies: not inside a capture).
int32_t batch_prepare(phx_batch b) {
    Ctx* c = b->ctx;
    const size_t nj = b->jobs.size();
    PHX_TRY(b->counters.reserve(nj * 3 * sizeof(unsigned long long)));
    PHX_TRY(b->stamps.reserve((nj + 1) * sizeof(unsigned long long)));
    PHX_TRY(b->next.reserve(4));
    PHX_TRY(b->modes.reserve(nj * 4));
    b->order.resize(nj);
    for (size_t j = 0; j < nj; j++) b->order[j] = (uint32_t)j;
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](uint32_t x, uint32_t y) { return b->jobs[x].spp > b->jobs[y].spp; });
    std::vector<Job> host(nj);
    uint32_t tile = 0;
    for (size_t k = 0; k < nj; k++) {
        const uint32_t j = b->order[k];
        BatchJob& bj = b->jobs[j];
        phx_tracer tr = bj.tr;
        PHX_TRY(ensure_image(tr, bj.w, bj.h));
        PHX_CUDA(cudaMemcpyAsync(tr->cam.ptr, &bj.cam, sizeof(phx_camera), cudaMemcpyHostToDevice, c->stream));
        Job& J = host[k];
        memset(&J, 0, sizeof J);
        J.S = scene_of(tr);
        J.S.smem_stack = b->stack == PHX_STACK_SHARED ? 1u : 0u;
        J.F = frame_for(tr, &bj.cam, bj.w, bj.h, bj.first, bj.spp);
        J.sun = mk(bj.cam.sun[0], bj.cam.sun[1], bj.cam.sun[2]);
        J.px = (uint32_t*)tr->px.ptr;
        J.counters = (unsigned long long*)b->counters.ptr + 3 * j;
        J.tile0 = tile;
        J.npx = bj.w * bj.h;
        tile += (J.npx + 31) / 32;
    }
    b->ntiles = tile;
    PHX_TRY(b->djobs.reserve(nj * sizeof(Job)));
    PHX_CUDA(cudaMemcpyAsync(b->djobs.ptr, host.data(), nj * sizeof(Job), cudaMemcpyHostToDevice, c->stream));
    return wait_stream(c->stream, BATCH_WAIT_MS);  // the pageable sources are released on return
}

// The frame's traces, stream-ordered (capturable once batch_prepare ran).
int32_t batch_trace(phx_batch b) {
    Ctx* c = b->ctx;
    PHX_CUDA(cudaMemsetAsync(b->counters.ptr, 0, b->jobs.size() * 3 * sizeof(unsigned long long), c->stream));
    if (b->kind == PHX_BATCH_PER_SCENE) {
        for (size_t j = 0; j < b->jobs.size(); j++) {
            BatchJob& bj = b->jobs[j];
            const Frame F = frame_for(bj.tr, &bj.cam, bj.w, bj.h, bj.first, bj.spp);
            PHX_CUDA(cudaMemsetAsync(bj.tr->rays.ptr, 0, 8, c->stream));
            PHX_TRY(launch_frame(bj.tr, F, mk(bj.cam.sun[0], bj.cam.sun[1], bj.cam.sun[2]), 0, bj.w * bj.h, false));
            PHX_CUDA(cudaMemcpyAsync((unsigned long long*)b->counters.ptr + 3 * j, bj.tr->rays.ptr, 8,
                                     cudaMemcpyDeviceToDevice, c->stream));
        }
        return PHX_OK;
    }
    switch (b->threads) {
        case 64: return launch_batch<64>(b);
        case 128: return launch_batch<128>(b);
        case 256: return launch_batch<256>(b);
    }
    return fail(PHX_ERR_INVALID, "batch block size %u (64, 128 or 256)", b->threads);
}

void batch_mark_traced(phx_batch b) {
    for (BatchJob& bj : b->jobs) {
        bj.tr->frame = bj.first + bj.spp - 1;
        bj.tr->last = bj.cam;
        bj.tr->have_last = true;
    }
}

void batch_drop_graph(phx_batch b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
}

int32_t clone_net(phx_ctx ctx, phx_unet src, phx_unet* out) {
    uint64_t count = 0;
    PHX_TRY(phx_unet_param_count(src, &count));
    std::vector<float> p(count);
    PHX_TRY(phx_unet_get(src, 0, p.data(), count));
    PHX_TRY(phx_unet_create(ctx, 1, out));
    const int32_t rc = phx_unet_set_params(*out, p.data(), count);
    if (rc < 0) {
        phx_unet_destroy(*out);
        *out = nullptr;
    }
    return rc;
}

}  // namespace
}  // namespace phx

extern "C" {

int32_t phx_batch_create(phx_ctx ctx, phx_batch* out) {
    if (!ctx || !out) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(&ctx->c));
    phx_batch b = new phx_batch_s();
    b->handle = ctx;
    b->ctx = &ctx->c;
    if (cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
        delete b;
        return fail(PHX_ERR_DEVICE, "event create");
    }
    ctx->c.live++;
    *out = b;
    return PHX_OK;
}

int32_t phx_batch_clear(phx_batch b) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    PHX_TRY(use(b->ctx));
    PHX_TRY(wait_stream(b->ctx->stream, BATCH_WAIT_MS));
    batch_drop_graph(b);
    for (phx_unet n : b->nets) phx_unet_destroy(n);
    b->nets.clear();
    b->net_of.clear();
    b->jobs.clear();
    b->ntiles = 0;
    return PHX_OK;
}

int32_t phx_batch_destroy(phx_batch b) {
    if (!b) return PHX_OK;
    phx_batch_clear(b);
    if (b->host_modes) cudaFreeHost(b->host_modes);
    if (b->done) cudaEventDestroy(b->done);
    b->ctx->live--;
    delete b;
    return PHX_OK;
}

int32_t phx_batch_add(phx_batch b, phx_tracer tr, const phx_camera* cam, uint32_t w, uint32_t h, uint32_t first,
                      uint32_t spp, uint32_t* index) {
    if (!b || !tr || !cam) return fail(PHX_ERR_INVALID, "null argument");
    if (tr->ctx != b->ctx) return fail(PHX_ERR_INVALID, "the tracer belongs to another context");
    if (w == 0 || h == 0 || spp == 0) return fail(PHX_ERR_INVALID, "empty job %ux%u x %u spp", w, h, spp);
    if ((uint64_t)w * h * PHX_PX_LEN + 1 > 0xFFFFFFFFull) return fail(PHX_ERR_INVALID, "image %ux%u too large", w, h);
    for (const BatchJob& bj : b->jobs)
        if (bj.tr == tr) return fail(PHX_ERR_INVALID, "a tracer can hold one job of a batch");
    PHX_TRY(check_camera(cam));
    if (tr->adapt[3] != 0.0f)
        return fail(PHX_ERR_INVALID, "adaptive sampling runs on single-scene traces (phx_tracer_trace/sample)");
    batch_drop_graph(b);
    b->jobs.push_back(BatchJob{tr, *cam, w, h, first, spp});
    std::memset(b->jobs.back().cam.adapt, 0, sizeof b->jobs.back().cam.adapt);  // the tracer's setting rules
    if (index) *index = (uint32_t)(b->jobs.size() - 1);
    return PHX_OK;
}

int32_t phx_batch_set_config(phx_batch b, uint32_t kind, uint32_t threads, uint32_t stack) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    if (kind > PHX_BATCH_PERSISTENT_DENSE) return fail(PHX_ERR_INVALID, "unknown batch kind %u", kind);
    if (threads != 64 && threads != 128 && threads != 256) return fail(PHX_ERR_INVALID, "block size %u", threads);
    if (stack > PHX_STACK_SHARED) return fail(PHX_ERR_INVALID, "stack placement %u", stack);
    batch_drop_graph(b);
    b->kind = kind;
    b->threads = threads;
    b->stack = stack;
    return PHX_OK;
}

int32_t phx_batch_trace(phx_batch b) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    if (b->jobs.empty()) return PHX_OK;
    PHX_TRY(use(b->ctx));
    PHX_TRY(batch_prepare(b));
    PHX_TRY(batch_trace(b));
    batch_mark_traced(b);
    return PHX_OK;
}

int32_t phx_batch_autotune(phx_batch b, uint32_t* kind, uint32_t* threads, uint32_t* stack, float* ms,
                           uint32_t* nconfigs) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    if (b->jobs.empty()) return fail(PHX_ERR_INVALID, "empty batch");
    PHX_TRY(use(b->ctx));
    struct Cfg {
        uint32_t kind, threads, stack, tracer_kernel;
    };
    std::vector<Cfg> cfgs;
    for (uint32_t t : {64u, 128u, 256u})
        for (uint32_t st : {PHX_STACK_LOCAL, PHX_STACK_SHARED}) cfgs.push_back({PHX_BATCH_PERSISTENT, t, st, 0});
    cfgs.push_back({PHX_BATCH_PER_SCENE, 128, PHX_STACK_LOCAL, PHX_KERNEL_MEGAKERNEL});
    cfgs.push_back({PHX_BATCH_PER_SCENE, 128, PHX_STACK_LOCAL, PHX_KERNEL_STATE_MACHINE});
    // every thread slot resident (32 registers): the single-scene winner's budget
    for (uint32_t t : {128u, 256u}) cfgs.push_back({PHX_BATCH_PERSISTENT_DENSE, t, PHX_STACK_LOCAL, 0});
    cfgs.push_back({PHX_BATCH_PER_SCENE, 128, PHX_STACK_LOCAL, PHX_KERNEL_MEGAKERNEL_16_SYNC});
    std::vector<uint32_t> saved;
    for (const BatchJob& bj : b->jobs) saved.push_back(bj.tr->kernel);
    cudaEvent_t e0, e1;
    PHX_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PHX_ERR_DEVICE, "event create");
    }
    float best = 3.0e38f;
    size_t pick = 0;
    int32_t rc = PHX_OK;
    for (size_t k = 0; k < cfgs.size() && rc == PHX_OK; k++) {
        const Cfg& cf = cfgs[k];
        b->kind = cf.kind;
        b->threads = cf.threads;
        b->stack = cf.stack;
        if (cf.kind == PHX_BATCH_PER_SCENE)
            for (BatchJob& bj : b->jobs) bj.tr->kernel = cf.tracer_kernel;
        if ((rc = batch_prepare(b)) < 0 || (rc = batch_trace(b)) < 0) break;  // warm-up
        cudaEventRecord(e0, b->ctx->stream);
        if ((rc = batch_trace(b)) < 0) break;
        cudaEventRecord(e1, b->ctx->stream);
        if ((rc = wait_stream(b->ctx->stream, BATCH_WAIT_MS)) < 0) break;
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (ms) ms[k] = t;
        if (t < best) {
            best = t;
            pick = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t j = 0; j < b->jobs.size(); j++)
        b->jobs[j].tr->kernel = cfgs[pick].kind == PHX_BATCH_PER_SCENE ? cfgs[pick].tracer_kernel : saved[j];
    PHX_TRY(rc);
    batch_drop_graph(b);
    b->kind = cfgs[pick].kind;
    b->threads = cfgs[pick].threads;
    b->stack = cfgs[pick].stack;
    if (kind) *kind = b->kind;
    if (threads) *threads = b->threads;
    if (stack) *stack = b->stack;
    if (nconfigs) *nconfigs = (uint32_t)cfgs.size();
    for (BatchJob& bj : b->jobs) bj.tr->have_last = false;  // the images hold tuning frames
    return read_status(b->ctx);
}

int32_t phx_batch_capture(phx_batch b, phx_unet net, float threshold) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    if (b->jobs.empty()) return fail(PHX_ERR_INVALID, "empty batch");
    for (const BatchJob& bj : b->jobs)
        if (bj.tr->forest || bj.tr->tree != PHX_TREE_LBVH)
            return fail(PHX_ERR_INVALID, "the serving graph rebuilds single-instance LBVH scenes; trace scenes "
                                         "of instances or on an SAH tree with phx_batch_trace");
    PHX_TRY(use(b->ctx));
    Ctx* c = b->ctx;
    PHX_TRY(wait_stream(c->stream, BATCH_WAIT_MS));
    batch_drop_graph(b);
    for (phx_unet n : b->nets) phx_unet_destroy(n);
    b->nets.clear();
    b->net_of.assign(b->jobs.size(), -1);
    PHX_TRY(batch_prepare(b));
    if (!b->host_modes) PHX_CUDA(cudaHostAlloc((void**)&b->host_modes, b->jobs.size() * 4, cudaHostAllocDefault));
    // One network per padded image shape (each holds buffers for its shape;
    // nothing may be allocated while the frame is recorded), and a first
    // frame outside the capture that sizes every scratch buffer.
    std::vector<std::pair<uint32_t, uint32_t>> shapes;
    const float strength[4] = {64.0f, 8.0f, 40.0f, 7.0f};
    for (size_t j = 0; j < b->jobs.size(); j++) {
        BatchJob& bj = b->jobs[j];
        if (net) {
            const std::pair<uint32_t, uint32_t> sh{(bj.h + 15) / 16, (bj.w + 15) / 16};
            size_t k = 0;
            while (k < shapes.size() && shapes[k] != sh) k++;
            if (k == shapes.size()) {
                shapes.push_back(sh);
                phx_unet cl = nullptr;
                PHX_TRY(clone_net(b->handle, net, &cl));
                b->nets.push_back(cl);
            }
            b->net_of[j] = (int)k;
        }
    }
    PHX_TRY(batch_trace(b));
    for (size_t j = 0; j < b->jobs.size(); j++) {
        BatchJob& bj = b->jobs[j];
        if (b->net_of[j] >= 0)
            PHX_TRY(phx_unet_denoise_px(b->nets[b->net_of[j]], (uint32_t*)bj.tr->px.ptr, nullptr, bj.w, bj.h,
                                        bj.cam.view, 16, threshold, 0, nullptr));
        else
            PHX_TRY(phx_denoise(b->handle, (uint32_t*)bj.tr->px.ptr, bj.w, bj.h, strength, bj.cam.view, 0));
    }
    PHX_TRY(wait_stream(c->stream, BATCH_WAIT_MS));
    PHX_TRY(read_status(c));

    cudaGraph_t graph = nullptr;
    PHX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = PHX_OK;
    auto step = [&](int32_t r) {
        if (rc == PHX_OK && r < 0) rc = r;
    };
    unsigned long long* stamps = (unsigned long long*)b->stamps.ptr;
    k_stamp<<<1, 1, 0, c->stream>>>(stamps);
    step(cuda_check(cudaMemcpyAsync(b->modes.ptr, b->host_modes, b->jobs.size() * 4, cudaMemcpyHostToDevice,
                                    c->stream), "modes"));
    for (size_t j = 0; j < b->jobs.size() && rc == PHX_OK; j++) {
        phx_tracer tr = b->jobs[j].tr;
        const uint32_t* mode = (const uint32_t*)b->modes.ptr + j;
        step(launch_face_boxes(c->stream, (const float*)tr->verts.ptr, (const uint32_t*)tr->faces.ptr, tr->nfaces,
                               (phx_aabb*)tr->bvh.prims.ptr));
        step(enqueue_build(c, tr->bvh, tr->nfaces, tr->leaf, Gate{mode, 1u}));
        step(enqueue_refit(c, tr->bvh, tr->nfaces, false, Gate{mode, 0u}));
        step(prepare(tr));
    }
    if (rc == PHX_OK) step(batch_trace(b));
    for (size_t j = 0; j < b->jobs.size() && rc == PHX_OK; j++) {
        BatchJob& bj = b->jobs[j];
        if (b->net_of[j] >= 0)
            step(phx_unet_denoise_px(b->nets[b->net_of[j]], (uint32_t*)bj.tr->px.ptr, nullptr, bj.w, bj.h,
                                     bj.cam.view, 16, threshold, 0, nullptr));
        else
            step(phx_denoise(b->handle, (uint32_t*)bj.tr->px.ptr, bj.w, bj.h, strength, bj.cam.view, 0));
        k_stamp<<<1, 1, 0, c->stream>>>(stamps + 1 + j);
    }
    const cudaError_t end = cudaStreamEndCapture(c->stream, &graph);
    if (rc == PHX_OK) rc = cuda_check(end, "end capture");
    if (rc == PHX_OK) rc = cuda_check(cudaGraphInstantiate(&b->exec, graph, 0), "instantiate frame graph");
    if (graph) cudaGraphDestroy(graph);
    if (rc < 0) batch_drop_graph(b);
    return rc;
}

int32_t phx_batch_replay(phx_batch b, const uint32_t* modes) {
    if (!b || !modes) return fail(PHX_ERR_INVALID, "null argument");
    if (!b->exec) return fail(PHX_ERR_INVALID, "no captured frame (phx_batch_capture)");
    PHX_TRY(use(b->ctx));
    // the previous replay has read its modes before they are overwritten
    PHX_TRY(wait_stream(b->ctx->stream, BATCH_WAIT_MS));
    for (size_t j = 0; j < b->jobs.size(); j++) b->host_modes[j] = modes[j] ? 1u : 0u;
    PHX_CUDA(cudaGraphLaunch(b->exec, b->ctx->stream));
    PHX_CUDA(cudaEventRecord(b->done, b->ctx->stream));
    batch_mark_traced(b);
    return PHX_OK;
}

int32_t phx_batch_results(phx_batch b, uint64_t* latency_ns, uint64_t* rays) {
    if (!b) return fail(PHX_ERR_INVALID, "null batch");
    PHX_TRY(use(b->ctx));
    PHX_TRY(wait_stream(b->ctx->stream, BATCH_WAIT_MS));
    const size_t nj = b->jobs.size();
    if (latency_ns && b->stamps.ptr) {
        std::vector<unsigned long long> st(nj + 1);
        PHX_CUDA(cudaMemcpy(st.data(), b->stamps.ptr, (nj + 1) * 8, cudaMemcpyDeviceToHost));
        for (size_t j = 0; j < nj; j++) latency_ns[j] = st[1 + j] - st[0];
    }
    if (rays && b->counters.ptr) {
        std::vector<unsigned long long> ct(nj * 3);
        PHX_CUDA(cudaMemcpy(ct.data(), b->counters.ptr, nj * 24, cudaMemcpyDeviceToHost));
        for (size_t j = 0; j < nj; j++) rays[j] = ct[3 * j];
    }
    return read_status(b->ctx);
}

}  // extern "C"
