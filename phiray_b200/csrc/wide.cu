// A 4-wide tree for ray-buffer walks, collapsed on the device from the
// binary tree the tracer walks (the LBVH or the binned SAH tree), and the
// persistent walk over it.
//
// Why: an incoherent ray in the binary walk spends most of its time in
// divergent, dependent two-box steps (about 16-21 of them a ray on the C2
// mesh). A 4-wide node holds four children's boxes, so a ray takes about
// half the steps, each with four independent slab tests, and the lanes of a
// warp reconverge twice as often per level of the tree.
//
// Collapse (top down, one level of wide nodes a launch): a wide node starts
// from a binary inner record (both children's boxes and refs) and opens
// its inner child with the largest surface area, twice at most, until it
// has four children or only leaves. Leaf refs (first slot | LEAF) are kept
// as they are, so a leaf is walked over the same triangle slots; each inner
// child becomes a wide node of the next level. Boxes are copied, not
// recomputed: the wide tree's boxes are the binary tree's.
//
// Record: 8 float4 = lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of children 0-3,
// their refs (NONE for an empty child), and a spare float4; 128 bytes.
//
// Results: closest hits are the binary walk's (the smallest t over the same
// triangles); only the order in which equal-t faces are met differs, so a
// tie between two faces at one t may name the other face. An any-hit ray
// reports hit or miss as the binary walk does.
#include "render.cuh"

namespace phx {

namespace {

using namespace shade;

__device__ __forceinline__ float half_area(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float dx = fmaxf(hx - lx, 0.0f), dy = fmaxf(hy - ly, 0.0f), dz = fmaxf(hz - lz, 0.0f);
    return dx * dy + dy * dz + dz * dx;
}

struct Child {
    float lo[3], hi[3];
    uint32_t ref;
};

// The two children of binary record r.
__device__ __forceinline__ void open_record(const float4* __restrict__ bin, uint32_t r, Child& a, Child& b) {
    const float4* q = bin + 4 * (size_t)r;
    const float4 n0 = __ldg(q), n1 = __ldg(q + 1), n2 = __ldg(q + 2), n3 = __ldg(q + 3);
    a = Child{{n0.x, n0.y, n0.z}, {n0.w, n1.x, n1.y}, __float_as_uint(n3.x)};
    b = Child{{n1.z, n1.w, n2.x}, {n2.y, n2.z, n2.w}, __float_as_uint(n3.y)};
}

// One level of the collapse: job k = (wide id, binary record).
__global__ void __launch_bounds__(128) k_wide_level(const float4* __restrict__ bin, const uint2* __restrict__ jobs,
                                                    uint32_t count, float4* __restrict__ wide, uint32_t* wcount,
                                                    uint2* __restrict__ next, uint32_t* next_count) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint2 job = jobs[k];
    Child c[4];
    int m = 2;
    open_record(bin, job.y, c[0], c[1]);
    for (int open = 0; open < 2; open++) {
        int pick = -1;
        float best = -1.0f;
        for (int j = 0; j < 4; j++) {
            if (j >= m || (c[j].ref & LEAF)) continue;
            const float a = half_area(c[j].lo[0], c[j].lo[1], c[j].lo[2], c[j].hi[0], c[j].hi[1], c[j].hi[2]);
            if (a > best) {
                best = a;
                pick = j;
            }
        }
        if (pick < 0) break;
        Child l, r;
        open_record(bin, c[pick].ref, l, r);
        // (m < 4 here: two opens from two children)
        for (int j = 0; j < 4; j++) {
            if (j == pick) c[j] = l;
            if (j == m) c[j] = r;
        }
        m++;
    }
    uint32_t inner = 0;
    for (int j = 0; j < 4; j++)
        if (j < m && !(c[j].ref & LEAF)) inner++;
    const uint32_t base = inner ? atomicAdd(wcount, inner) : 0u;
    const uint32_t at = inner ? atomicAdd(next_count, inner) : 0u;
    float v[6][4];
    uint32_t ref[4];
    uint32_t t = 0;
    for (int j = 0; j < 4; j++) {
        if (j < m) {
            for (int e = 0; e < 3; e++) {
                v[2 * e][j] = c[j].lo[e];
                v[2 * e + 1][j] = c[j].hi[e];
            }
            if (c[j].ref & LEAF) {
                ref[j] = c[j].ref;
            } else {
                ref[j] = base + t;
                next[at + t] = make_uint2(base + t, c[j].ref);
                t++;
            }
        } else {
            for (int e = 0; e < 3; e++) {
                v[2 * e][j] = 0.0f;
                v[2 * e + 1][j] = 0.0f;
            }
            ref[j] = NONE;
        }
    }
    float4* o = wide + 8 * (size_t)job.x;
    for (int r = 0; r < 6; r++) o[r] = make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
    o[6] = make_float4(__uint_as_float(ref[0]), __uint_as_float(ref[1]), __uint_as_float(ref[2]),
                       __uint_as_float(ref[3]));
    o[7] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

template <bool ANY, bool STATS>
__global__ void __launch_bounds__(128, 8) k_rays_wide_thread(Scene S, const float4* __restrict__ wide,
                                                             const float4* __restrict__ rays, uint32_t n,
                                                             float4* __restrict__ hits,
                                                             unsigned long long* counters) {
    load_info(S);
    const Tree T = tree_of(S);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count cnt{0, 0, 0};
    if (i < n) {
        const float4 a = __ldg(rays + 2 * (size_t)i), b = __ldg(rays + 2 * (size_t)i + 1);
        const Hit h = walk_wide<STATS>(T, wide, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, ANY, cnt);
        const uint32_t face = h.tri == NONE ? NONE : __float_as_uint(__ldg(T.tris + 3 * (size_t)h.tri).w);
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

constexpr int WIDE_STEPS = 20;  // visits a round: 12-24 swept on the C2 bounce rays, 20 fastest

// k_rays_fetch's persistent warps over the wide tree: each lane walks one
// ray nearest child first (four slab tests a step, the hit children sorted
// by entry distance), and idle lanes take the next rays from a counter
// between rounds of WIDE_STEPS visits. (A two-phase round, every lane
// stepping inner nodes until all hold a leaf, then the leaves together, ran
// 8 % slower on the C2 mesh's bounce rays.)
template <bool ANY, bool STATS>
__global__ void __launch_bounds__(128, 8) k_rays_wide(Scene S, const float4* __restrict__ wide,
                                                      const float4* __restrict__ rays, uint32_t n,
                                                      float4* __restrict__ hits, unsigned long long* counters,
                                                      uint32_t* next) {
    load_info(S);
    const Tree T = tree_of(S);
    const uint32_t root = (T.root & LEAF) ? T.root : 0u;
    const int lane = threadIdx.x & 31;
    Count cnt{0, 0, 0};
    uint32_t stack[WSTACK];
    bool active = false;
    uint32_t idx = 0, nd = 0;
    int sp = 0;
    f3 o = mk(0.0f), inv = mk(0.0f);
    RaySpace rs;
    rs.kz = 2u;
    rs.flip = false;
    rs.s = mk(0.0f);
    Hit best{0.0f, NONE, 0.0f, 0.0f, 0u};
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
                    const float4 a = __ldg(rays + 2 * (size_t)idx), b = __ldg(rays + 2 * (size_t)idx + 1);
                    o = mk(a.x, a.y, a.z);
                    const f3 d = mk(b.x, b.y, b.z);
                    cnt.rays++;
                    best = Hit{a.w, NONE, 0.0f, 0.0f, 0u};
                    inv = safe_inv(d);
                    rs = ray_space(d);
                    sp = 0;
                    nd = root;
                    active = box_t(T.root_lo, T.root_hi, o, inv, best.t) < INF;
                    if (!active) hits[idx] = make_float4(best.t, __uint_as_float(NONE), 0.0f, 0.0f);
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) {
            uint32_t seen = 0;
            if (lane == 0) seen = atomicAdd(next, 0u);
            seen = __shfl_sync(0xffffffffu, seen, 0);
            if (seen >= n) break;
            continue;
        }
        for (int it = 0; it < WIDE_STEPS && active; it++) {
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
                                best = Hit{t, id, u, v, 0u};
                                done = true;
                                break;
                            }
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
                // sort the four (t, ref) pairs by t: a 5-comparator network
                order2(t0, r0, t1, r1);
                order2(t2, r2, t3, r3);
                order2(t0, r0, t2, r2);
                order2(t1, r1, t3, r3);
                order2(t1, r1, t2, r2);
                if (t0 < INF) {
                    // farthest first, so the nearest of the rest is on top
                    if (t3 < INF && sp < WSTACK) stack[sp++] = r3;
                    if (t2 < INF && sp < WSTACK) stack[sp++] = r2;
                    if (t1 < INF && sp < WSTACK) stack[sp++] = r1;
                    nd = r0;
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
    if (STATS) {
        const uint32_t st = __reduce_add_sync(0xffffffffu, cnt.steps);
        const uint32_t te = __reduce_add_sync(0xffffffffu, cnt.tests);
        if (lane == 0) {
            atomicAdd(counters + 1, (unsigned long long)st);
            atomicAdd(counters + 2, (unsigned long long)te);
        }
    }
}

}  // namespace

int32_t build_wide(const float4* bin, uint32_t ninner, float4* wide, uint2* jobs_a, uint2* jobs_b, uint32_t* counts,
                   cudaStream_t s, uint32_t* nodes_out, uint32_t* levels_out) {
    // counts[0]: wide nodes handed out; counts[1]: the next level's jobs
    *nodes_out = 0;
    *levels_out = 0;
    if (ninner == 0) return PHX_OK;
    const uint32_t one[2] = {1u, 0u};
    const uint2 first = make_uint2(0u, 0u);
    PHX_CUDA(cudaMemcpyAsync(counts, one, 8, cudaMemcpyHostToDevice, s));
    PHX_CUDA(cudaMemcpyAsync(jobs_a, &first, 8, cudaMemcpyHostToDevice, s));
    uint32_t len = 1, levels = 0;
    while (len) {
        if (levels >= 64) return fail(PHX_ERR_DEVICE, "wide tree: more than 64 levels");
        PHX_CUDA(cudaMemsetAsync(counts + 1, 0, 4, s));
        k_wide_level<<<(len + 127) / 128, 128, 0, s>>>(bin, jobs_a, len, wide, counts, jobs_b, counts + 1);
        PHX_CUDA(cudaGetLastError());
        uint32_t got[2] = {0, 0};
        PHX_CUDA(cudaMemcpyAsync(got, counts, 8, cudaMemcpyDeviceToHost, s));
        PHX_CUDA(cudaStreamSynchronize(s));
        if (got[0] > ninner) return fail(PHX_ERR_DEVICE, "wide tree: more nodes than binary inner nodes");
        len = got[1];
        std::swap(jobs_a, jobs_b);
        levels++;
        *nodes_out = got[0];
    }
    *levels_out = levels;
    return PHX_OK;
}

int32_t launch_rays_wide(const Scene& S, const float4* wide, const float* rays, uint32_t n, float* hits, bool any,
                         unsigned long long* counters, uint32_t* next, int sms, cudaStream_t s) {
    if (!next) {  // a thread a ray
        const uint32_t blocks = (n + 127) / 128;
        const float4* R = (const float4*)rays;
        float4* H = (float4*)hits;
        if (any) {
            if (counters) k_rays_wide_thread<true, true><<<blocks, 128, 0, s>>>(S, wide, R, n, H, counters);
            else k_rays_wide_thread<true, false><<<blocks, 128, 0, s>>>(S, wide, R, n, H, counters);
        } else {
            if (counters) k_rays_wide_thread<false, true><<<blocks, 128, 0, s>>>(S, wide, R, n, H, counters);
            else k_rays_wide_thread<false, false><<<blocks, 128, 0, s>>>(S, wide, R, n, H, counters);
        }
        return cuda_check(cudaGetLastError(), "wide ray walk");
    }
    int per_sm = 0;
    const bool st = counters != nullptr;
    if (any) {
        if (st) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rays_wide<true, true>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rays_wide<true, false>, 128, 0);
    } else {
        if (st) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rays_wide<false, true>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rays_wide<false, false>, 128, 0);
    }
    const uint32_t grid = std::min<uint32_t>((uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sms, (n + 127) / 128);
    PHX_CUDA(cudaMemsetAsync(next, 0, 4, s));
    const float4* R = (const float4*)rays;
    float4* H = (float4*)hits;
    if (any) {
        if (st) k_rays_wide<true, true><<<grid, 128, 0, s>>>(S, wide, R, n, H, counters, next);
        else k_rays_wide<true, false><<<grid, 128, 0, s>>>(S, wide, R, n, H, counters, next);
    } else {
        if (st) k_rays_wide<false, true><<<grid, 128, 0, s>>>(S, wide, R, n, H, counters, next);
        else k_rays_wide<false, false><<<grid, 128, 0, s>>>(S, wide, R, n, H, counters, next);
    }
    return cuda_check(cudaGetLastError(), "wide ray walk");
}

}  // namespace phx
