// The Rendered path's device code: the LBVH walk and the bounce loop.
//
// Reference: src/trace/wgsl/bvh.wgsl (box_t, ray_space, tri_t, safe_inv,
// trace_blas/trace), shade.wgsl main (:41-373), integrate.wgsl (direct,
// indirect, glow_mis, bounce_light, cosine_dir), light.wgsl (onb, cone_dir,
// env_at, visible, lamp_query, area_query, spot_mask, lamp_reach,
// lamp_chance, glow_query, hit_lift, through_lift), brdf.wgsl (GGX, Surf,
// fresnel_of, dielectric_f0, under_layer(_real), env_brdf, brdf_w,
// ggx_pdf, glossy_floor), util.wgsl (hash, rnd, unit_disk), view.wgsl.
//
// A scene is either one identity instance (every mesh in world space: the
// reference's top-tree walk plus one trace_blas is then a single walk of the
// mesh tree, in the same order: root box, near child first, strict
// `t < best`), or meshes placed by instances: a top tree over the instances'
// world boxes, each leaf's instances walked in turn with the ray taken into
// the mesh's space by the instance's inverse (bvh.wgsl trace, trace_blas).
// Features the tracer does not take (textures, procedural slots,
// environment images, depth of field, film transparency) are refused on the
// host.
//
// Layout the walk reads (built from the LBVH after every build/refit):
//   nodes  4 float4 per inner node: both children's boxes, then their refs
//          (inner node index, or first slot | LEAF)
//   tris   3 float4 per sorted slot: a.xyz + face id, b.xyz + material id,
//          c.xyz + flags (bit 0: last slot of its leaf; bit 1: a shadow
//          ray passes it — glass or cut-out, bvh.wgsl:158-162)
// so one step is one 64-byte node read and one triangle one 48-byte read.
// With instances the top tree's records come first (a leaf ref is
// first top slot | LEAF | INST), then each mesh's; inst_slots[s] names top
// slot s's instance (END on the last slot of a leaf), and each instance is a
// record of 8 float4: the world matrix's rows (3), its inverse's rows (3),
// the mesh's root box lo with the root ref in .w, and hi with the flags in
// .w (bit 0 at the identity, 1 casts no shadow, 2 mirrors).
#pragma once

#include "internal.cuh"
#include "vec.cuh"

namespace phx {
namespace shade {

constexpr uint32_t LEAF = 0x80000000u;
constexpr uint32_t INST = 0x40000000u;      // a top-tree leaf: its range is instance slots (forest.rs INST)
constexpr uint32_t INST_END = 0x80000000u;  // the last slot of a top-tree leaf (inst_slots)
constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr float INF = 3.0e38f;
constexpr float PI = 3.14159265f;
constexpr uint32_t FLAG_END = 1u;
constexpr uint32_t FLAG_PASS = 2u;
constexpr int STACK = 32;

struct Scene {
    const float4* __restrict__ nodes;
    const float4* __restrict__ tris;
    const float4* __restrict__ tnorm;  // 3 per slot, or null: flat faces
    const float4* __restrict__ mats;   // 8 float4 (32 words, trace::Mat) per material
    const uint32_t* __restrict__ lamp_slot;
    const float* __restrict__ lamp_cdf;
    const float4* __restrict__ info;   // root box + ref, extent, emitter count (device results of the build)
    const float4* __restrict__ insts;  // instance records, or null: one identity instance
    const uint32_t* __restrict__ inst_slots;  // top slot -> instance (| INST_END)
    const uint32_t* __restrict__ lamp_inst;   // the emitter table's instance column (instanced scenes)
    uint32_t nslots;  // triangles: a leaf walk never reads past them
    uint32_t lamp_count;
    uint32_t root;  // inner node 0, or LEAF | 0 when the root is a leaf
    f3 root_lo, root_hi;
    float extent;
    // The walks' 32-entry stacks: per-thread local memory (0), or (1) this
    // thread's column of the launch's dynamic shared memory, which must then
    // hold 32 words per thread.
    uint32_t smem_stack;
};

// Fills the build-dependent fields from the device info record, and the
// frame's ray offsets from the extent (Tracer::sample_in, sample.rs:114-118:
// ao = 8% of the extent when the camera leaves it 0, eps = 1e-5 of it).
__device__ __forceinline__ void load_info(Scene& S) {
    const float4 a = __ldg(S.info), b = __ldg(S.info + 1), c = __ldg(S.info + 2);
    S.root_lo = mk(a.x, a.y, a.z);
    S.root = __float_as_uint(a.w);
    S.root_hi = mk(b.x, b.y, b.z);
    S.extent = b.w;
    S.lamp_count = __float_as_uint(c.x);
}

struct Hit {
    float t;
    uint32_t tri;  // sorted slot, NONE for a miss
    float u, v;
    uint32_t inst;  // the instance the hit came through (0 for one identity instance)
};

// Rays traced by a thread, and (STATS builds) the walk's node steps and
// triangle tests — the work the walk's bytes are counted from.
struct Count {
    uint32_t rays, steps, tests;
};

// Render modes, a kernel's compile-time int template argument: bit 0 counts
// node steps and triangle tests (STATS builds); bit 1 (FULL) takes scenes of
// instances and draws the floor grid overlay. Kernels without it take
// single-instance scenes with the grid off — every benchmark frame — and
// hold no two-level walk, placed geometry or grid code.
constexpr int MODE_STATS = 1;
constexpr int MODE_FULL = 2;
constexpr int MODE_ANY = MODE_FULL;  // code that takes any scene
// Bits 2 and 3 place the single-instance walk's stack: its top entry (REG)
// or top 8 entries (REG | REG8) in registers, the rest in local memory.
constexpr int MODE_REG = 4;
constexpr int MODE_REG8 = 8;

// Where a walk keeps its 32-entry stack: a per-thread local array, this
// thread's column of a block-wide shared array, or a short stack of R
// registers over a local array (place REG_BASE + R).
constexpr int PLACE_LOCAL = 0;
constexpr int PLACE_SHARED = 1;
constexpr int PLACE_REG_BASE = 16;
template <int M>
constexpr int PLACE_OF_MODE = (M & MODE_REG) ? PLACE_REG_BASE + ((M & MODE_REG8) ? 8 : 1) : PLACE_LOCAL;

struct Frame {
    uint32_t w, h, n, frame0, spp, persp, count, bounces;
    f3 right, up, back, pivot, env;
    float scale, units, aspect, dist, pan_x, pan_y, ao, eps;  // ao: the camera's (0 = auto); eps set in-kernel
    float sky[4];
    float limit_d, limit_i, exposure, gamma;
    const phx_light* __restrict__ lights;
    // Adaptive Sampling (util.wgsl:61-99): on, the convergence threshold,
    // the minimum samples and the step; `list`: this launch traces the
    // open-pixel list (px word 32n + k, its length at 34n) instead of
    // pixel k.
    uint32_t adapt_on, adapt_min, adapt_step, adapt_list;
    float adapt_thr;
    // The floor grid overlay (util.wgsl:185-272): Camera.grid (0 = off),
    // grid_color, grid_hide.
    float grid;
    float4 grid_color;
    uint32_t grid_hide;
};

// ---- util.wgsl ----

__device__ __forceinline__ uint32_t hash(uint32_t x) {
    uint32_t h = x * 747796405u + 2891336453u;
    h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
    return (h >> 22u) ^ h;
}

__device__ __forceinline__ float rnd(uint32_t& seed) {
    seed = hash(seed);
    return (float)seed / 4294967295.0f;
}

__device__ __forceinline__ float2 unit_disk(float ru, float rv) {
    const float a = 2.0f * ru - 1.0f;
    const float b = 2.0f * rv - 1.0f;
    if (a == 0.0f && b == 0.0f) return make_float2(0.0f, 0.0f);
    float r, phi;
    if (a * a > b * b) {
        r = a;
        phi = (PI / 4.0f) * (b / a);
    } else {
        r = b;
        phi = (PI / 2.0f) - (PI / 4.0f) * (a / b);
    }
    float s, c;
    pm_sincos(phi, &s, &c);
    return make_float2(r * c, r * s);
}

// ---- bvh.wgsl ----

__device__ __forceinline__ float box_t(f3 lo, f3 hi, f3 o, f3 inv, float best) {
    const f3 t1 = (lo - o) * inv;
    const f3 t2 = (hi - o) * inv;
    const float tmin = fmaxf(fmaxf(fminf(t1.x, t2.x), fminf(t1.y, t2.y)), fminf(t1.z, t2.z));
    const float tmax = fminf(fminf(fmaxf(t1.x, t2.x), fmaxf(t1.y, t2.y)), fmaxf(t1.z, t2.z));
    if (tmax >= fmaxf(tmin, 0.0f) && tmin < best) return fmaxf(tmin, 0.0f);
    return INF;
}

struct RaySpace {
    uint32_t kz;
    bool flip;
    f3 s;
};

__device__ __forceinline__ f3 ray_axes(f3 v, uint32_t kz, bool flip) {
    const f3 p = kz == 2u ? v : (kz == 0u ? mk(v.y, v.z, v.x) : mk(v.z, v.x, v.y));
    return flip ? mk(p.y, p.x, p.z) : p;
}

__device__ __forceinline__ RaySpace ray_space(f3 d) {
    const f3 a = mk(fabsf(d.x), fabsf(d.y), fabsf(d.z));
    const uint32_t kz = (a.x >= a.y && a.x >= a.z) ? 0u : (a.y >= a.z ? 1u : 2u);
    const bool flip = ray_axes(d, kz, false).z < 0.0f;
    const f3 dr = ray_axes(d, kz, flip);
    const float sz = 1.0f / dr.z;
    return RaySpace{kz, flip, mk(dr.x * sz, dr.y * sz, sz)};
}

// Watertight test (Woop et al. 2013): t, or INF for a miss; u, v the
// weights of tb and tc.
__device__ __forceinline__ float tri_t(f3 ta, f3 tb, f3 tc, f3 o, const RaySpace& r, float& u, float& v) {
    const f3 a = ray_axes(ta - o, r.kz, r.flip);
    const f3 b = ray_axes(tb - o, r.kz, r.flip);
    const f3 c = ray_axes(tc - o, r.kz, r.flip);
    const float ax = a.x - r.s.x * a.z;
    const float ay = a.y - r.s.y * a.z;
    const float bx = b.x - r.s.x * b.z;
    const float by = b.y - r.s.y * b.z;
    const float cx = c.x - r.s.x * c.z;
    const float cy = c.y - r.s.y * c.z;
    const float ea = cx * by - cy * bx;
    const float eb = ax * cy - ay * cx;
    const float ec = bx * ay - by * ax;
    if ((ea < 0.0f || eb < 0.0f || ec < 0.0f) && (ea > 0.0f || eb > 0.0f || ec > 0.0f)) return INF;
    const float det = ea + eb + ec;
    if (det == 0.0f) return INF;
    const float tt = ea * (r.s.z * a.z) + eb * (r.s.z * b.z) + ec * (r.s.z * c.z);
    const float sg = det < 0.0f ? -1.0f : 1.0f;
    if (tt * sg <= 0.0f) return INF;
    const float inv = 1.0f / det;
    u = eb * inv;
    v = ec * inv;
    return tt * inv;
}

__device__ __forceinline__ f3 safe_inv(f3 d) {
    const float sx = d.x < 0.0f ? -1.0f : 1.0f, sy = d.y < 0.0f ? -1.0f : 1.0f, sz = d.z < 0.0f ? -1.0f : 1.0f;
    return mk(1.0f / (fabsf(d.x) < 1e-9f ? sx * 1e-9f : d.x), 1.0f / (fabsf(d.y) < 1e-9f ? sy * 1e-9f : d.y),
              1.0f / (fabsf(d.z) < 1e-9f ? sz * 1e-9f : d.z));
}

__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }

// trace (bvh.wgsl:120-232) over the single-instance tree. `first`: any hit
// (a shadow ray), which passes glass and cut-outs and stops at the first
// opaque hit. The stack holds 32 refs; the builder caps the depth at 31.
// The arrays and root a walk reads, passed by value so they stay in
// registers across the walk loop (a reference to a struct in local memory is
// re-read every step when the loop's stack stores might alias it).
struct Tree {
    const float4* __restrict__ nodes;
    const float4* __restrict__ tris;
    uint32_t nslots, root;
    f3 root_lo, root_hi;
};

__device__ __forceinline__ Tree tree_of(const Scene& S) {
    return Tree{S.nodes, S.tris, S.nslots, S.root, S.root_lo, S.root_hi};
}

// The traversal stack at placement P: a per-thread array in local memory,
// this thread's column of a block-wide shared array (entry k at
// shared[k * stride]), or a short stack whose top R entries sit in registers
// and whose older entries spill to a local array. Every placement pops in
// the same last-in first-out order and holds at most STACK entries (a push
// onto a full stack is dropped), so the walk visits the same nodes.
template <int P, bool REG = (P >= PLACE_REG_BASE)>
struct Stack {
    static constexpr int SPILL = 1;  // the caller's spill array: unused here
    uint32_t local[P == PLACE_SHARED ? 1 : STACK];
    uint32_t* shared;
    int stride;
    int sp = 0;
    __device__ __forceinline__ void bind(uint32_t*, uint32_t* smem, int smem_stride) {
        shared = smem;
        stride = smem_stride;
    }
    __device__ __forceinline__ bool empty() const { return sp == 0; }
    __device__ __forceinline__ void push(uint32_t x) {
        if (sp >= STACK) return;
        if (P == PLACE_SHARED) shared[sp++ * stride] = x;
        else local[sp++] = x;
    }
    __device__ __forceinline__ uint32_t pop() {
        sp--;
        return P == PLACE_SHARED ? shared[sp * stride] : local[sp];
    }
};

// The register placement keeps its spill array outside the struct (the
// caller's local array), so the struct's own fields stay in registers. A
// pop refills the registers from the spill array at once, so that load's
// latency passes while the popped subtree is walked.
template <int P>
struct Stack<P, true> {
    static constexpr int R = P - PLACE_REG_BASE;
    static constexpr int SPILL = STACK - R;
    uint32_t reg[R];
    uint32_t* spill;
    int sp = 0;  // entries in the spill array
    int nr = 0;  // entries in registers
    __device__ __forceinline__ void bind(uint32_t* s, uint32_t*, int) { spill = s; }
    __device__ __forceinline__ bool empty() const { return sp + nr == 0; }
    __device__ __forceinline__ void push(uint32_t x) {
        if (sp + nr >= STACK) return;
        // the oldest register entry spills once all R are held
        if (nr == R) spill[sp++] = reg[R - 1];
        else nr++;
#pragma unroll
        for (int k = R - 1; k > 0; k--) reg[k] = reg[k - 1];
        reg[0] = x;
    }
    __device__ __forceinline__ uint32_t pop() {
        const uint32_t x = reg[0];
#pragma unroll
        for (int k = 0; k < R - 1; k++) reg[k] = reg[k + 1];
        // the spill array holds entries only while every register is full
        if (sp > 0) reg[R - 1] = spill[--sp];
        else nr--;
        return x;
    }
};

// One tree's walk from its root (box test first), improving `best`; true
// when an any-hit ray found its opaque hit. Hits record `inst`.
template <bool STATS, int P = PLACE_LOCAL>
__device__ __forceinline__ bool walk_tree(const Tree S, f3 o, f3 d, Hit& best, bool first, uint32_t inst, Count& cnt,
                                          uint32_t* smem_stack = nullptr, int stride = 0) {
    const f3 inv = safe_inv(d);
    if (box_t(S.root_lo, S.root_hi, o, inv, best.t) >= INF) return false;
    const RaySpace rs = ray_space(d);
    uint32_t spill[Stack<P>::SPILL];
    Stack<P> stack;
    stack.bind(spill, smem_stack, stride);
    uint32_t nd = S.root;
    for (;;) {
        if (nd & LEAF) {
            for (uint32_t id = nd & ~LEAF; id < S.nslots; id++) {
                const float4 A = __ldg(S.tris + 3 * (size_t)id);
                const float4 B = __ldg(S.tris + 3 * (size_t)id + 1);
                const float4 Cc = __ldg(S.tris + 3 * (size_t)id + 2);
                const uint32_t flags = __float_as_uint(Cc.w);
                if (STATS) cnt.tests++;
                float u, v;
                const float t = tri_t(xyz(A), xyz(B), xyz(Cc), o, rs, u, v);
                if (t < best.t) {
                    if (first) {
                        if (!(flags & FLAG_PASS)) {
                            best = Hit{t, id, u, v, inst};
                            return true;
                        }
                    } else {
                        best = Hit{t, id, u, v, inst};
                    }
                }
                if (flags & FLAG_END) break;
            }
        } else {
            if (STATS) cnt.steps++;
            const float4* q = S.nodes + 4 * (size_t)nd;
            const float4 n0 = __ldg(q), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3);
            const float tl = box_t(mk(n0.x, n0.y, n0.z), mk(n0.w, n1.x, n1.y), o, inv, best.t);
            const float tr = box_t(mk(n1.z, n1.w, n2.x), mk(n2.y, n2.z, n2.w), o, inv, best.t);
            const uint32_t l = __float_as_uint(n3.x), r = __float_as_uint(n3.y);
            if (tl < INF && tr < INF) {
                // Depth <= 31 keeps the stack below STACK entries; push's
                // check only guards a corrupt tree from writing past it.
                stack.push(tl <= tr ? r : l);
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
        if (stack.empty()) break;
        nd = stack.pop();
    }
    return false;
}

// A ray's walk of a single-instance scene's tree.
template <bool STATS, int P = PLACE_LOCAL>
__device__ __forceinline__ Hit walk(const Tree S, f3 o, f3 d, float tmax, bool first, Count& cnt,
                                    uint32_t* smem_stack = nullptr, int stride = 0) {
    cnt.rays++;
    Hit best{tmax, NONE, 0.0f, 0.0f, 0u};
    walk_tree<STATS, P>(S, o, d, best, first, 0u, cnt, smem_stack, stride);
    return best;
}

__device__ __forceinline__ float row_point(float4 r, f3 p) { return ((r.x * p.x + r.y * p.y) + r.z * p.z) + r.w * 1.0f; }
__device__ __forceinline__ float row_dir(float4 r, f3 d) { return (r.x * d.x + r.y * d.y) + r.z * d.z; }

// trace_blas (bvh.wgsl:115-190): instance i's mesh tree, walked in the mesh's
// space (the ray taken there by the instance's inverse, its direction left
// unnormalised so t is the world's); a shadow ray passes an instance that
// casts none. True when an any-hit ray found its hit.
template <bool STATS, int P>
__device__ __forceinline__ bool walk_instance(const Scene& S, uint32_t i, f3 ow, f3 dw, Hit& best, bool first,
                                              Count& cnt, uint32_t* smem_stack, int stride) {
    const float4* q = S.insts + 8 * (size_t)i;
    const float4 lo = __ldg(q + 6), hi = __ldg(q + 7);
    const uint32_t root = __float_as_uint(lo.w), flags = __float_as_uint(hi.w);
    if (root == NONE) return false;
    if (first && (flags & 2u)) return false;
    f3 o = ow, d = dw;
    if (!(flags & 1u)) {
        const float4 i0 = __ldg(q + 3), i1 = __ldg(q + 4), i2 = __ldg(q + 5);
        o = mk(row_point(i0, ow), row_point(i1, ow), row_point(i2, ow));
        d = mk(row_dir(i0, dw), row_dir(i1, dw), row_dir(i2, dw));
    }
    const Tree T{S.nodes, S.tris, S.nslots, root, xyz(lo), xyz(hi)};
    return walk_tree<STATS, P>(T, o, d, best, first, i, cnt, smem_stack, stride);
}

// trace (bvh.wgsl:194-232) over a scene of instances: the top tree over
// their world boxes, near child first; at a leaf each of its instances'
// trees in slot order; an any-hit ray stops at its first hit. The top
// walk's stack is a second 32-entry stack (the reference's trace and
// trace_blas each keep one).
template <bool STATS, int P = PLACE_LOCAL>
__device__ __forceinline__ Hit walk_forest(const Scene& S, f3 o, f3 d, float tmax, bool first, Count& cnt,
                                           uint32_t* smem_stack = nullptr, int stride = 0) {
    cnt.rays++;
    Hit best{tmax, NONE, 0.0f, 0.0f, 0u};
    const f3 inv = safe_inv(d);
    if (box_t(S.root_lo, S.root_hi, o, inv, best.t) >= INF) return best;
    uint32_t stack[STACK];
    int sp = 0;
    uint32_t nd = S.root;
    for (;;) {
        if (nd & LEAF) {
            for (uint32_t s = nd & ~(LEAF | INST);; s++) {
                const uint32_t e = __ldg(S.inst_slots + s);
                if (walk_instance<STATS, P>(S, e & ~INST_END, o, d, best, first, cnt, smem_stack, stride))
                    return best;
                if (e & INST_END) break;
            }
        } else {
            if (STATS) cnt.steps++;
            const float4* q = S.nodes + 4 * (size_t)nd;
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
        if (sp == 0) break;
        sp--;
        nd = stack[sp];
    }
    return best;
}

// ---- the 4-wide tree of the ray-buffer walks (wide.cu builds it from the
// binary records; inside the 32-register render kernels its larger frame
// cost more than its fewer steps saved, so the frame walks stay binary) ----
// Record: 8 float4 = lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of children 0-3,
// their refs (inner wide record, first slot | LEAF, or NONE), a spare.

constexpr int WSTACK = 96;  // 3 pushes a wide level, 31 levels at most

__device__ __forceinline__ void order2(float& ta, uint32_t& ra, float& tb, uint32_t& rb) {
    if (tb < ta) {
        const float t = ta;
        ta = tb;
        tb = t;
        const uint32_t r = ra;
        ra = rb;
        rb = r;
    }
}

// One ray's walk of the wide tree: each node's hit children sorted by entry
// distance (a 5-comparator network), the nearest taken, the rest pushed
// farthest first. `first`: any hit, as walk_tree. The closest t equals the
// binary walk's; only which face a tie of two faces at one t names may
// differ.
template <bool STATS>
__device__ __forceinline__ Hit walk_wide(const Tree& T, const float4* __restrict__ wide, f3 o, f3 d, float tmax,
                                         bool first, Count& cnt) {
    cnt.rays++;
    Hit best{tmax, NONE, 0.0f, 0.0f, 0u};
    const f3 inv = safe_inv(d);
    if (box_t(T.root_lo, T.root_hi, o, inv, best.t) >= INF) return best;
    const RaySpace rs = ray_space(d);
    uint32_t stack[WSTACK];
    int sp = 0;
    uint32_t nd = (T.root & LEAF) ? T.root : 0u;
    for (;;) {
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
                    if (first) {
                        if (!(flags & FLAG_PASS)) return Hit{t, id, u, v, 0u};
                    } else {
                        best = Hit{t, id, u, v, 0u};
                    }
                }
                if (flags & FLAG_END) break;
            }
        } else {
            if (STATS) cnt.steps++;
            const float4* q = wide + 8 * (size_t)nd;
            const float4 lx = __ldg(q), hx = __ldg(q + 1), ly = __ldg(q + 2), hy = __ldg(q + 3);
            const float4 lz = __ldg(q + 4), hz = __ldg(q + 5), rf = __ldg(q + 6);
            uint32_t r0 = __float_as_uint(rf.x), r1 = __float_as_uint(rf.y);
            uint32_t r2 = __float_as_uint(rf.z), r3 = __float_as_uint(rf.w);
            float t0 = box_t(mk(lx.x, ly.x, lz.x), mk(hx.x, hy.x, hz.x), o, inv, best.t);
            float t1 = box_t(mk(lx.y, ly.y, lz.y), mk(hx.y, hy.y, hz.y), o, inv, best.t);
            float t2 = r2 == NONE ? INF : box_t(mk(lx.z, ly.z, lz.z), mk(hx.z, hy.z, hz.z), o, inv, best.t);
            float t3 = r3 == NONE ? INF : box_t(mk(lx.w, ly.w, lz.w), mk(hx.w, hy.w, hz.w), o, inv, best.t);
            order2(t0, r0, t1, r1);
            order2(t2, r2, t3, r3);
            order2(t0, r0, t2, r2);
            order2(t1, r1, t3, r3);
            order2(t1, r1, t2, r2);
            if (t0 < INF) {
                if (t3 < INF && sp < WSTACK) stack[sp++] = r3;
                if (t2 < INF && sp < WSTACK) stack[sp++] = r2;
                if (t1 < INF && sp < WSTACK) stack[sp++] = r1;
                nd = r0;
                continue;
            }
        }
        if (sp == 0) break;
        nd = stack[--sp];
    }
    return best;
}

// The two-level walk behind a call of its own, so a single-instance scene's
// trace keeps a frame of one stack.
template <bool STATS>
__device__ __noinline__ Hit trace_forest(const Scene& S, f3 o, f3 d, float tmax, bool first, Count& cnt) {
    if (S.smem_stack) {
        extern __shared__ uint32_t walk_stacks[];
        return walk_forest<STATS, PLACE_SHARED>(S, o, d, tmax, first, cnt, walk_stacks + threadIdx.x, (int)blockDim.x);
    }
    return walk_forest<STATS>(S, o, d, tmax, first, cnt);
}

// A ray's walk of either kind of scene.
template <bool STATS, int P = PLACE_LOCAL>
__device__ __forceinline__ Hit walk_scene(const Scene& S, f3 o, f3 d, float tmax, bool first, Count& cnt,
                                          uint32_t* smem_stack = nullptr, int stride = 0) {
    if (S.insts) return trace_forest<STATS>(S, o, d, tmax, first, cnt);
    return walk<STATS, P>(tree_of(S), o, d, tmax, first, cnt, smem_stack, stride);
}

// A ray's walk in a render mode: the two-level walk only where the mode
// takes instances and the scene has them.
template <int M>
__device__ __forceinline__ Hit walk_mode(const Scene& S, f3 o, f3 d, float tmax, bool first, Count& cnt) {
    constexpr bool STATS = (M & MODE_STATS) != 0;
    if ((M & MODE_FULL) && S.insts) return trace_forest<STATS>(S, o, d, tmax, first, cnt);
    return walk<STATS, PLACE_OF_MODE<M>>(tree_of(S), o, d, tmax, first, cnt);
}

// The walk behind a call, for code with several trace sites.
template <int M>
__device__ __noinline__ Hit trace(const Scene& S, f3 o, f3 d, float tmax, bool first, Count& cnt) {
    constexpr bool STATS = (M & MODE_STATS) != 0;
    if ((M & MODE_FULL) && S.insts) return trace_forest<STATS>(S, o, d, tmax, first, cnt);
    if constexpr ((M & MODE_REG) != 0) {
        return walk<STATS, PLACE_OF_MODE<M>>(tree_of(S), o, d, tmax, first, cnt);
    } else {
        if (S.smem_stack) {
            extern __shared__ uint32_t walk_stacks[];
            return walk<STATS, PLACE_SHARED>(tree_of(S), o, d, tmax, first, cnt, walk_stacks + threadIdx.x,
                                             (int)blockDim.x);
        }
        return walk<STATS>(tree_of(S), o, d, tmax, first, cnt);
    }
}

// ---- scene records ----

struct Mat {
    float4 color;
    float rough, metal, trans, ior;
    f3 emit;
    float sss;
    f3 sss_radius;
    float sheen, sheen_rough;
    f3 sheen_tint;
    float coat, coat_rough;
};

__device__ __forceinline__ Mat mat_at(const Scene& S, uint32_t m) {
    const float4* q = S.mats + 8 * (size_t)m;
    const float4 w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2), w4 = __ldg(q + 4), w5 = __ldg(q + 5),
                 w6 = __ldg(q + 6);
    Mat t;
    t.color = w0;
    t.rough = w1.x;
    t.metal = w1.y;
    t.trans = w1.z;
    t.ior = w1.w;
    t.emit = mk(w2.x, w2.y, w2.z);
    t.sss = w4.y;
    t.sss_radius = mk(w4.z, w4.w, w5.x);
    t.sheen = w5.y;
    t.sheen_rough = w5.z;
    t.sheen_tint = mk(w5.w, w6.x, w6.y);
    t.coat = w6.z;
    t.coat_rough = w6.w;
    return t;
}

struct Geo {
    f3 a, b, c, na, nb, nc;
    uint32_t face, mat;
    bool mirror;  // placed by a mirroring instance: world_ng turns the face normal back
};

// place_n (layout.wgsl:72-77): a normal under the inverse-transpose of an
// instance's 3 x 3, unit again; a zero (flat) normal stays zero.
__device__ __forceinline__ f3 place_n(float4 i0, float4 i1, float4 i2, f3 n) {
    const f3 m = xyz(i0) * n.x + xyz(i1) * n.y + xyz(i2) * n.z;
    const float l = length(m);
    if (l < 1e-12f) return mk(0.0f);
    return m / l;
}

// tri_of (layout.wgsl:114-159): the face in `slot`, placed in the world by
// instance `inst` (vertices are kept in the mesh's space, w = 1) in a mode
// that takes instances.
template <int M>
__device__ __forceinline__ Geo geo_at(const Scene& S, uint32_t slot, uint32_t inst) {
    const float4 A = __ldg(S.tris + 3 * (size_t)slot), B = __ldg(S.tris + 3 * (size_t)slot + 1),
                 Cc = __ldg(S.tris + 3 * (size_t)slot + 2);
    Geo g;
    g.a = xyz(A);
    g.b = xyz(B);
    g.c = xyz(Cc);
    g.face = __float_as_uint(A.w);
    g.mat = __float_as_uint(B.w);
    if (S.tnorm) {
        g.na = xyz(__ldg(S.tnorm + 3 * (size_t)slot));
        g.nb = xyz(__ldg(S.tnorm + 3 * (size_t)slot + 1));
        g.nc = xyz(__ldg(S.tnorm + 3 * (size_t)slot + 2));
    } else {
        g.na = g.nb = g.nc = mk(0.0f);
    }
    g.mirror = false;
    if ((M & MODE_FULL) && S.insts) {
        const float4* q = S.insts + 8 * (size_t)inst;
        const uint32_t flags = __float_as_uint(__ldg(q + 7).w);
        g.mirror = (flags & 4u) != 0u;
        if (!(flags & 1u)) {
            const float4 r0 = __ldg(q), r1 = __ldg(q + 1), r2 = __ldg(q + 2);
            g.a = mk(row_point(r0, g.a), row_point(r1, g.a), row_point(r2, g.a));
            g.b = mk(row_point(r0, g.b), row_point(r1, g.b), row_point(r2, g.b));
            g.c = mk(row_point(r0, g.c), row_point(r1, g.c), row_point(r2, g.c));
            const float4 i0 = __ldg(q + 3), i1 = __ldg(q + 4), i2 = __ldg(q + 5);
            g.na = place_n(i0, i1, i2, g.na);
            g.nb = place_n(i0, i1, i2, g.nb);
            g.nc = place_n(i0, i1, i2, g.nc);
        }
    }
    return g;
}

// ---- brdf.wgsl ----

struct Surf {
    f3 pos, n, v, albedo, f0;
    float rough, bleed;
    f3 sss_tint;
    float sheen, sheen_rough;
    f3 sheen_tint;
    float coat, coat_rough, eta, dielectric;
};

__device__ __forceinline__ float ggx_lambda(float alpha2, float cos_n) {
    const float t = alpha2 * fmaxf(1.0f / fmaxf(cos_n * cos_n, 1e-8f) - 1.0f, 0.0f);
    return 0.5f * (sqrtf(1.0f + t) - 1.0f);
}

__device__ __forceinline__ f3 ggx_sample_vndf(f3 wi, float alpha, float r1, float r2) {
    const f3 wi_ = normalize(mk(alpha * wi.x, alpha * wi.y, wi.z));
    const float lensq = wi_.x * wi_.x + wi_.y * wi_.y;
    f3 t1, t2;
    if (lensq > 1e-7f) {
        t1 = mk(-wi_.y, wi_.x, 0.0f) / sqrtf(lensq);
        t2 = cross(wi_, t1);
    } else {
        t1 = mk(1.0f, 0.0f, 0.0f);
        t2 = mk(0.0f, 1.0f, 0.0f);
    }
    float2 t = unit_disk(r1, r2);
    t.y = mixf(sqrtf(fmaxf(1.0f - t.x * t.x, 0.0f)), t.y, 0.5f * (1.0f + wi_.z));
    const f3 h_ = t1 * t.x + t2 * t.y + wi_ * sqrtf(fmaxf(0.0f, 1.0f - t.x * t.x - t.y * t.y));
    return normalize(mk(alpha * h_.x, alpha * h_.y, fmaxf(0.0f, h_.z)));
}

__device__ __forceinline__ float ggx_weight(float alpha2, float cos_ni, float cos_no) {
    const float li = ggx_lambda(alpha2, cos_ni);
    const float lo = ggx_lambda(alpha2, cos_no);
    return (1.0f + li) / (1.0f + li + lo);
}

__device__ __forceinline__ Surf plain_surf(f3 pos, f3 n, f3 v, f3 albedo, f3 f0, float rough) {
    return Surf{pos, n, v, albedo, f0, rough, 0.0f, mk(1.0f), 0.0f, 0.5f, mk(1.0f), 0.0f, 0.03f, 0.0f, 0.0f};
}

// procedural.wgsl:73-81
__device__ __forceinline__ float fresnel_dielectric_cos(float cosi, float eta) {
    const float c = fabsf(cosi);
    float g = eta * eta - 1.0f + c * c;
    if (g <= 0.0f) return 1.0f;
    g = sqrtf(g);
    const float a = (g - c) / (g + c);
    const float b = (c * (g + c) - 1.0f) / (c * (g - c) + 1.0f);
    return 0.5f * a * a * (1.0f + b * b);
}

__device__ __forceinline__ f3 fresnel_of(const Surf& s, float cs) {
    const float schlick = pm_pow(1.0f - cs, 5.0f);
    f3 f = s.f0 + (mk(1.0f) - s.f0) * schlick;
    if (s.eta > 1.0f && s.dielectric > 0.0f) {
        const float r = (s.eta - 1.0f) / (s.eta + 1.0f);
        const float face_on = r * r;
        f += mk(s.dielectric * (fresnel_dielectric_cos(cs, s.eta) - face_on - (1.0f - face_on) * schlick));
    }
    return vmax(f, mk(0.0f));
}

__device__ __forceinline__ f3 scatter_tint(f3 radius) {
    const float m = fmaxf(fmaxf(radius.x, radius.y), fmaxf(radius.z, 1e-6f));
    return vmix(mk(1.0f), radius / m, 0.85f);
}

__device__ __forceinline__ float scatter_bleed(float weight, f3 radius) {
    const float m = fmaxf(fmaxf(radius.x, radius.y), fmaxf(radius.z, 0.0f));
    return clampf(weight, 0.0f, 1.0f) * clampf(m * 24.0f, 0.15f, 1.0f);
}

__device__ __forceinline__ float charlie(float nh, float rough) {
    const float inv = 1.0f / fmaxf(rough * rough, 0.005f);
    const float sin2 = fmaxf(1.0f - nh * nh, 0.0f);
    return (2.0f + inv) * pm_pow(sin2, inv * 0.5f) / (2.0f * PI);
}

__device__ __forceinline__ f3 env_brdf(f3 f0, float rough, float nv) {
    const float rx = rough * -1.0f + 1.0f, ry = rough * -0.0275f + 0.0425f, rz = rough * -0.572f + 1.04f,
                rw = rough * 0.022f + -0.04f;
    const float a004 = fminf(rx * rx, pm_exp2(-9.28f * nv)) * rx + ry;
    const float abx = -1.04f * a004 + rz, aby = 1.04f * a004 + rw;
    return f0 * abx + mk(aby);
}

__device__ __forceinline__ f3 dielectric_f0(float ior) {
    const float r = (ior - 1.0f) / (ior + 1.0f);
    return mk(r * r);
}

__device__ __forceinline__ float under_layer(f3 f0, float rough, float nv) {
    const f3 e = env_brdf(f0, rough, nv);
    return clampf(1.0f - fmaxf(e.x, fmaxf(e.y, e.z)), 0.0f, 1.0f);
}

__device__ __forceinline__ float under_layer_real(float eta, float rough, float nv) {
    const float r = (eta - 1.0f) / (eta + 1.0f);
    const float face_on = r * r;
    const float climb = env_brdf(mk(0.0f), rough, nv).x;
    const float flat = env_brdf(mk(1.0f), rough, nv).x - climb;
    const float schlick = (1.0f - face_on) * pm_pow(1.0f - nv, 5.0f);
    const float real = fresnel_dielectric_cos(nv, eta) - face_on;
    const float scale = clampf(real / fmaxf(schlick, 1e-5f), 0.0f, 1.0f);
    return clampf(1.0f - (face_on * flat + climb * scale), 0.0f, 1.0f);
}

// glossy_floor with phiray's own integrator (integrator.x 0): 0.3.
__device__ __forceinline__ float glossy_floor() { return 0.3f; }

__device__ __forceinline__ float ggx_pdf(const Surf& s, f3 l) {
    const f3 h = normalize(l + s.v);
    const float nh = fmaxf(dot(s.n, h), 0.0f);
    const float a2 = fmaxf(s.rough * s.rough * s.rough * s.rough, 1e-4f);
    const float dd = nh * nh * (a2 - 1.0f) + 1.0f;
    const float dist = a2 / (PI * dd * dd);
    const float nv = fmaxf(dot(s.n, s.v), 1e-4f);
    const float g1 = 1.0f / (1.0f + ggx_lambda(a2, nv));
    return g1 * dist / (4.0f * nv);
}

__device__ __forceinline__ f3 brdf_w(const Surf& s, f3 l, f3 e, float wd, float ws) {
    const float raw = dot(s.n, l);
    const float w = s.bleed * 0.75f;
    const float nl = fmaxf((raw + w) / (1.0f + w), 0.0f) / (1.0f + w * 0.5f);
    f3 thru = mk(0.0f);
    if (s.bleed != 0.0f) thru = s.albedo * s.bleed * s.sss_tint * pm_pow(fmaxf(dot(s.v, -l), 0.0f), 3.0f) * 0.35f;
    if (nl <= 0.0f) return thru * e * wd;
    const f3 hv = normalize(l + s.v);
    const float nh = fmaxf(dot(s.n, hv), 0.0f);
    const float hvv = fmaxf(dot(hv, s.v), 0.0f);
    const float a2 = fmaxf(s.rough * s.rough * s.rough * s.rough, 1e-4f);
    const float dd = nh * nh * (a2 - 1.0f) + 1.0f;
    const float dist = a2 / (PI * dd * dd);
    const f3 fres = fresnel_of(s, hvv);
    const float nv = fmaxf(dot(s.n, s.v), 1e-4f);
    const float g2 = 1.0f / (1.0f + ggx_lambda(a2, nv) + ggx_lambda(a2, fmaxf(raw, 1e-4f)));
    const f3 spec = fres * dist * g2 * 0.25f / nv;
    const f3 diffuse = vmix(s.albedo, s.albedo * s.sss_tint, s.bleed) / PI;
    f3 sum = diffuse * wd + spec * ws;
    if (s.sheen != 0.0f) sum += s.sheen_tint * s.sheen * charlie(nh, s.sheen_rough);
    if (s.coat != 0.0f) {
        const float ca2 = fmaxf(s.coat_rough * s.coat_rough * s.coat_rough * s.coat_rough, 1e-4f);
        const float cd = nh * nh * (ca2 - 1.0f) + 1.0f;
        const float coat_f = 0.04f + 0.96f * pm_pow(1.0f - hvv, 5.0f);
        const float coat = s.coat * coat_f * (ca2 / (PI * cd * cd)) * 0.25f;
        const float under = 1.0f - s.coat * coat_f;
        sum = sum * under + mk(coat);
    }
    f3 out = sum * e * nl;
    if (s.bleed != 0.0f) out += thru * e * wd;
    return out;
}

__device__ __forceinline__ f3 brdf(const Surf& s, f3 l, f3 e) { return brdf_w(s, l, e, 1.0f, 1.0f); }

// ---- light.wgsl ----

__device__ __forceinline__ f3 onb(f3 n, float a, float b) {
    const f3 tx = normalize(fabsf(n.z) > 0.9f ? cross(n, mk(1.0f, 0.0f, 0.0f)) : cross(n, mk(0.0f, 0.0f, 1.0f)));
    const f3 ty = cross(n, tx);
    return tx * a + ty * b;
}

__device__ __forceinline__ f3 cone_dir(f3 axis, float ang, uint32_t& seed) {
    if (ang <= 0.0f) return axis;
    const float r = ang * sqrtf(rnd(seed));
    const float ph = 2.0f * PI * rnd(seed);
    float s, c;
    pm_sincos(ph, &s, &c);
    return normalize(axis + onb(axis, r * c, r * s));
}

__device__ __forceinline__ f3 cosine_dir(f3 n, uint32_t& seed) {
    const float r1 = rnd(seed);
    const float rr = sqrtf(r1);
    const float ph = 2.0f * PI * rnd(seed);
    float s, c;
    pm_sincos(ph, &s, &c);
    return normalize(onb(n, rr * c, rr * s) + n * sqrtf(fmaxf(0.0f, 1.0f - r1)));
}

struct Shadowed {
    f3 c, dir;
    float dist;
};

__device__ __forceinline__ Shadowed unshadowed() { return Shadowed{mk(0.0f), mk(0.0f, 0.0f, 1.0f), 0.0f}; }

__device__ __forceinline__ float spot_mask(const phx_light& li, f3 l) {
    const f3 dir = mk(li.dir[0], li.dir[1], li.dir[2]);
    const float z = -dot(l, dir);
    if (z <= 0.0f) return 0.0f;
    float ellipse = z;
    const f3 right = mk(li.right[0], li.right[1], li.right[2]);
    const float ssx = li.spot_scale[0], ssy = li.spot_scale[1];
    if (dot(right, right) > 1e-12f && ssx * ssx + ssy * ssy > 1e-12f) {
        const f3 d = -l;
        const float xx = dot(d, right) * ssx, yy = dot(d, cross(dir, right)) * ssy;
        ellipse = 1.0f / sqrtf(1.0f + (xx * xx + yy * yy) / (z * z));
    }
    return smoothstepf(li.cone, li.cone + li.blend, ellipse);
}

__device__ __forceinline__ float lamp_reach(const phx_light& li, f3 at, float ao) {
    const f3 color = mk(li.color[0], li.color[1], li.color[2]);
    const float lum = dot(vmax(color, mk(0.0f)), mk(0.2126f, 0.7152f, 0.0722f));
    if (li.kind == 0u) return lum;
    const f3 to = mk(li.pos[0], li.pos[1], li.pos[2]) - at;
    const float nr = fmaxf(li.size * 0.5f, ao * 0.05f);
    return lum / ((4.0f * PI) * (dot(to, to) + nr * nr));
}

__device__ __forceinline__ Shadowed area_query(const Surf& s, const phx_light& li, float weight, float r1, float r2,
                                               float pick) {
    const f3 lpos = mk(li.pos[0], li.pos[1], li.pos[2]), ldir = mk(li.dir[0], li.dir[1], li.dir[2]),
             lright = mk(li.right[0], li.right[1], li.right[2]);
    const float height = dot(s.pos - lpos, ldir);
    if (height <= 0.0f) return unshadowed();
    const bool round = li.shape == 4u || li.shape == 5u;
    const float hx = li.size * 0.5f, hy = li.size_y * 0.5f;
    const float area = fmaxf(li.size * li.size_y * (round ? 0.25f * PI : 1.0f), 1e-8f);
    const f3 up = cross(ldir, lright);
    const f3 off = s.pos - lpos;
    const float near = area / (area + PI * dot(off, off));
    float onx, ony;
    float sn, cs;
    pm_sincos(2.0f * PI * r2, &sn, &cs);
    if (pick < near) {
        const float spread = sqrtf(r1 / fmaxf(1.0f - r1, 1e-6f)) * height;
        onx = cs * spread + dot(off, lright);
        ony = sn * spread + dot(off, up);
        const float ux = onx / fmaxf(hx, 1e-8f), uy = ony / fmaxf(hy, 1e-8f);
        const bool inside = round ? (ux * ux + uy * uy <= 1.0f) : (fmaxf(fabsf(ux), fabsf(uy)) <= 1.0f);
        if (!inside) return unshadowed();
    } else {
        const float sq = sqrtf(r1);
        if (round) {
            onx = cs * sq * hx;
            ony = sn * sq * hy;
        } else {
            onx = (r1 * 2.0f - 1.0f) * hx;
            ony = (r2 * 2.0f - 1.0f) * hy;
        }
    }
    const f3 to = lpos + lright * onx + up * ony - s.pos;
    const float d2 = fmaxf(dot(to, to), 1e-6f);
    const f3 l = to / sqrtf(d2);
    const float facing = fmaxf(dot(-l, ldir), 0.0f);
    const float pdf = (1.0f - near) / area + near * facing * facing / (PI * d2);
    const f3 e = mk(li.color[0], li.color[1], li.color[2]) / (PI * area) * facing / d2 / fmaxf(pdf, 1e-12f);
    if (maxc(e) < 1e-5f) return unshadowed();
    return Shadowed{brdf(s, l, e) * weight, l, sqrtf(d2) * 0.999f};
}

__device__ __forceinline__ Shadowed lamp_query(const Frame& F, const Surf& s, uint32_t& seed) {
    float total = 0.0f, held = 0.0f;
    uint32_t idx = 0;
    float u = rnd(seed);
    for (uint32_t k = 0; k < F.count; k++) {
        const float w = lamp_reach(F.lights[k], s.pos, F.ao);
        if (w <= 0.0f) continue;
        total += w;
        const float share = w / total;
        if (u < share) {
            idx = k;
            held = w;
            u = u / share;
        } else {
            u = (u - share) / (1.0f - share);
        }
    }
    if (total <= 0.0f || held <= 0.0f) return unshadowed();
    const phx_light& li = F.lights[idx];
    const float weight = total / held;
    const f3 color = mk(li.color[0], li.color[1], li.color[2]);
    if (li.kind == 0u) {
        const f3 l = cone_dir(-mk(li.dir[0], li.dir[1], li.dir[2]), li.size * 0.5f, seed);
        return Shadowed{brdf(s, l, color) * weight, l, INF};
    }
    const float r1 = rnd(seed);
    const float r2 = rnd(seed);
    if (li.kind == 3u) return area_query(s, li, weight, r1, r2, rnd(seed));
    const f3 lpos = mk(li.pos[0], li.pos[1], li.pos[2]);
    const f3 aim = lpos + onb(normalize(s.pos - lpos), (r1 - 0.5f) * li.size, (r2 - 0.5f) * li.size);
    const f3 to = aim - s.pos;
    const float d2 = fmaxf(dot(to, to), 1e-6f);
    const f3 l = to / sqrtf(d2);
    f3 e = color / ((4.0f * PI) * d2);
    if (li.kind == 2u) e *= spot_mask(li, l);
    if (maxc(e) < 1e-5f) return unshadowed();
    return Shadowed{brdf(s, l, e) * weight, l, sqrtf(d2) * 0.999f};
}

// lamp_chance (light.wgsl:259-271): the table share of the hit's (face,
// instance) pair, the entries sorted by face, then instance.
template <int M>
__device__ __forceinline__ float lamp_chance(const Scene& S, uint32_t slot, uint32_t inst) {
    const uint32_t count = S.lamp_count;
    if (count == 0u) return 0.0f;
    const bool placed = (M & MODE_FULL) && S.lamp_inst;
    uint32_t lo = 0, hi = count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2u;
        const uint32_t f = __ldg(S.lamp_slot + mid);
        const uint32_t i = placed ? __ldg(S.lamp_inst + mid) : 0u;
        if (f < slot || (f == slot && i < inst)) lo = mid + 1u;
        else hi = mid;
    }
    if (__ldg(S.lamp_slot + lo) != slot || (placed ? __ldg(S.lamp_inst + lo) : 0u) != inst) return 0.0f;
    const float prev = lo > 0u ? __ldg(S.lamp_cdf + lo - 1u) : 0.0f;
    return __ldg(S.lamp_cdf + lo) - prev;
}

template <int M>
__device__ __forceinline__ Shadowed glow_query(const Scene& S, const Surf& s, uint32_t& seed) {
    const uint32_t count = S.lamp_count;
    if (count == 0u) return unshadowed();
    const float u = rnd(seed);
    uint32_t lo = 0, hi = count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2u;
        if (__ldg(S.lamp_cdf + mid) < u) lo = mid + 1u;
        else hi = mid;
    }
    const float prev = lo > 0u ? __ldg(S.lamp_cdf + lo - 1u) : 0.0f;
    const float chance = fmaxf(__ldg(S.lamp_cdf + lo) - prev, 1e-8f);
    const uint32_t f = __ldg(S.lamp_slot + lo);
    const Geo g = geo_at<M>(S, f, ((M & MODE_FULL) && S.lamp_inst) ? __ldg(S.lamp_inst + lo) : 0u);
    const Mat t = mat_at(S, g.mat);
    float a = rnd(seed);
    float b = rnd(seed);
    if (a + b > 1.0f) {
        a = 1.0f - a;
        b = 1.0f - b;
    }
    const f3 q = g.a + (g.b - g.a) * a + (g.c - g.a) * b;
    const f3 cr = cross(g.b - g.a, g.c - g.a);
    const float area = 0.5f * length(cr);
    const f3 to = q - s.pos;
    const float d2 = fmaxf(dot(to, to), 1e-6f);
    const f3 l = to / sqrtf(d2);
    const float cos_l = fabsf(dot(normalize(cr), l));
    const f3 e = t.emit * cos_l * area / (chance * d2);
    const float pl = chance * d2 / fmaxf(area * cos_l, 1e-8f);
    const float pb = fmaxf(dot(s.n, l), 0.0f) / PI;
    const float w = pl * pl / fmaxf(pl * pl + pb * pb, 1e-12f);
    return Shadowed{brdf(s, l, e) * w, l, sqrtf(d2) * 0.999f};
}

__device__ __forceinline__ float hit_lift(const Frame& F, float t) {
    const float start = 1.0e4f / F.units;
    if (F.persp == 0u && t > start * 0.5f) return F.eps + fabsf(t - start) * 1e-5f + start * 2.4e-7f;
    return F.eps + t * 1e-5f;
}

__device__ __forceinline__ float through_lift(const Frame& F, f3 pos, float t) {
    const float reach = fmaxf(fmaxf(fabsf(pos.x), fabsf(pos.y)), fmaxf(fabsf(pos.z), 0.5f));
    return hit_lift(F, t) - F.eps + reach * (256.0f / 8388608.0f);
}

__device__ __forceinline__ bool uses_rig(const Frame& F) { return F.count == 0u && !(dot(F.env, F.env) > 0.0f); }

__device__ __forceinline__ Shadowed rig_query(const Frame& F, uint32_t k, const Surf& s, uint32_t& seed, f3 sun) {
    if (k == 0u) {
        const f3 key = cone_dir(sun, 0.06f, seed);
        return Shadowed{brdf(s, key, mk(2.0f)), key, INF};
    }
    const f3 rim = normalize(F.up * 0.6f - F.back * 0.8f + F.right * 0.2f);
    return Shadowed{brdf(s, rim, mk(0.9f)), rim, INF};
}

// ---- util.wgsl:185-272: the floor grid as an overlay, premultiplied ----

struct Over {
    f3 c;
    float a;
};

// floor_over: Blender's floor grid on z = 0 (lines every power of ten, the
// finer level fading as its cells shrink, anti-aliased over one pixel's
// footprint, faded toward the horizon) and its X and Y axes.
__device__ __forceinline__ Over floor_over(const Frame& F, f3 o, f3 d, float t_hit, float px) {
    if (F.grid <= 0.0f || fabsf(d.z) < 1e-6f) return Over{mk(0.0f), 0.0f};
    const float t = -o.z / d.z;
    if (t <= 0.0f || t >= t_hit) return Over{mk(0.0f), 0.0f};
    const f3 q = o + d * t;
    float foot = px;
    if (F.persp != 0u) foot = px * t * F.units / F.dist;
    const float want = foot * 24.0f;
    const float lg = pm_log2(fmaxf(want, 1e-9f)) / pm_log2(10.0f);
    const float lvl = floorf(lg);
    const float f = lg - lvl;
    const float g0 = pm_pow(10.0f, lvl);
    const float g1 = g0 * 10.0f;
    const float half_w = foot * 0.5f;
    const float aa = foot;
    const float c0x = q.x / g0, c0y = q.y / g0, c1x = q.x / g1, c1y = q.y / g1;
    // WGSL round(): to nearest, ties to even, as rintf
    const float d0x = fabsf(c0x - rintf(c0x)) * g0, d0y = fabsf(c0y - rintf(c0y)) * g0;
    const float d1x = fabsf(c1x - rintf(c1x)) * g1, d1y = fabsf(c1y - rintf(c1y)) * g1;
    const float l0 = fmaxf(1.0f - smoothstepf(half_w, half_w + aa, d0x), 1.0f - smoothstepf(half_w, half_w + aa, d0y));
    const float l1 = fmaxf(1.0f - smoothstepf(half_w, half_w + aa, d1x), 1.0f - smoothstepf(half_w, half_w + aa, d1y));
    const float fine = (1.0f - f) * (1.0f - f);
    const float line = fmaxf(l0 * fine * 0.6f, l1);
    const float horizon = clampf(fabsf(d.z) * 4.0f, 0.0f, 1.0f);
    float depth = 1.0f;
    if (F.persp != 0u) {
        const float r = t * F.units / (F.dist * 6.0f);
        depth = 1.0f / (1.0f + r * r);
    }
    const float fade = horizon * depth;
    const float w0 = line * F.grid_color.w * fade * ((F.grid_hide & 1u) != 0u ? 0.0f : 1.0f);
    f3 c = mk(F.grid_color.x, F.grid_color.y, F.grid_color.z) * w0;
    float a = w0;
    const float ax = 1.0f - smoothstepf(half_w, half_w + aa, fabsf(q.y));
    const float ay = 1.0f - smoothstepf(half_w, half_w + aa, fabsf(q.x));
    const float w1 = ax * 0.85f * fade * ((F.grid_hide & 2u) != 0u ? 0.0f : 1.0f);
    c = c * (1.0f - w1) + mk(0.85f, 0.3f, 0.33f) * w1;
    a = a * (1.0f - w1) + w1;
    const float w2 = ay * 0.85f * fade * ((F.grid_hide & 4u) != 0u ? 0.0f : 1.0f);
    c = c * (1.0f - w2) + mk(0.47f, 0.72f, 0.2f) * w2;
    a = a * (1.0f - w2) + w2;
    return Over{c, a};
}

// z_axis_over: the vertical line through the origin, within half a pixel.
__device__ __forceinline__ Over z_axis_over(const Frame& F, f3 o, f3 d, float t_hit, float px) {
    const float a = d.x * d.x + d.y * d.y;
    if (a < 1e-12f) return Over{mk(0.0f), 0.0f};
    const float t = -(o.x * d.x + o.y * d.y) / a;
    if (t <= 0.0f || t >= t_hit) return Over{mk(0.0f), 0.0f};
    float foot = px;
    if (F.persp != 0u) foot = px * t * F.units / F.dist;
    const f3 at = o + d * t;
    const float r = sqrtf(at.x * at.x + at.y * at.y);
    const float w = (1.0f - smoothstepf(foot * 0.5f, foot * 1.5f, r)) * 0.85f;
    return Over{mk(0.25f, 0.53f, 0.92f) * w, w};
}

// grid_over: nothing unless the camera turns the grid on.
static __device__ __noinline__ Over grid_over(const Frame& F, f3 o, f3 d, float t_hit) {
    const float px = 1.0f / (F.scale * F.units * (float)F.w);
    Over g = floor_over(F, o, d, t_hit, px);
    if (F.grid > 0.0f && (F.grid_hide & 8u) != 0u) {
        const Over z = z_axis_over(F, o, d, t_hit, px);
        g = Over{g.c * (1.0f - z.a) + z.c, g.a * (1.0f - z.a) + z.a};
    }
    return g;
}

__device__ __forceinline__ f3 rig_fill(const Frame& F, const Surf& s) {
    const f3 fill = normalize(-F.right * 0.8f + F.up * 0.2f + F.back * 0.6f);
    return brdf(s, fill, mk(0.45f));
}

}  // namespace shade
}  // namespace phx
