// LBVH on the device, bit for bit the tree phiray's CPU builder makes.
//
// Reference: src/bvh/build.rs (Bvh::build: codes, sort_codes, Link::of,
// assemble, refit), src/bvh/node.rs (Node, Half, Aabb, morton),
// src/bvh/mod.rs (code, delta), src/bvh/gpu.rs (GpuBvh), and the WGSL
// kernels in src/bvh/kernel.rs. The reference's GpuBvh reads the Karras
// links and the order back and packs leaves on the CPU; here every stage
// stays on the device:
//
//   k_bounds        scene box partials (Bvh::scene, build.rs:70-72)
//   k_morton_hist   finish the box, 30-bit codes (build.rs:75-85), and the
//                   four 8-bit digit histograms of the radix sort
//   k_radix_pass x4 stable onesweep LSD passes: warp match ranks in shared
//                   memory, decoupled look-back across tiles, staged
//                   coalesced scatter. Stable, so the result equals the
//                   CPU's sort by (code, index) (build.rs:87-92).
//   k_karras        Link::of (build.rs:28-60) + parent pointers
//   k_pack          Bvh::assemble (build.rs:139-168) without a DFS: a node
//                   is a packed leaf iff cand(i) && !cand(parent(i)), where
//                   cand = (last - first < leaf) || depth + 1 >= STACK; cand
//                   holds for every descendant of a cand node, so that rule
//                   reproduces the DFS exactly. Depth = climb of parents.
//   k_refit         Bvh::refit (build.rs:180-194) as one atomic bottom-up
//                   pass: reachable leaves compute their box, the second
//                   child to arrive at a parent computes the parent's.
//
// min/max add no rounding, so codes, order, links, depth and bounds match
// the CPU builder exactly.
#include <cfloat>

#include "lbvh.cuh"

namespace phx {
namespace {

constexpr uint32_t LEAF = 0x80000000u;
constexpr uint32_t STACK = 32;
constexpr uint32_t NONE = 0xFFFFFFFFu;

constexpr int RADIX_THREADS = 256;
constexpr int RADIX_ITEMS = 16;
constexpr int TILE = RADIX_THREADS * RADIX_ITEMS;
constexpr int WARPS = RADIX_THREADS / 32;
constexpr int PASSES = 4;
static_assert(TILE == LBVH_TILE && PASSES == LBVH_PASSES, "lbvh.cuh and bvh.cu agree");
constexpr uint32_t FLAG_AGG = LOOKBACK_AGG;
constexpr uint32_t FLAG_INC = LOOKBACK_INC;
constexpr uint32_t VALUE_MASK = LOOKBACK_VALUE;
constexpr uint32_t SPIN_LIMIT = 1u << 22;
constexpr uint32_t MAX_PRIMS = 1u << 30;  // look-back words hold 30-bit counts

// morton's spread (node.rs:98-104; WGSL kernel.rs:33-39). fmaxf(NaN, 0) is
// 0, as Rust's `NaN as u64` is.
__device__ __forceinline__ uint32_t spread(float v) {
    uint32_t x = (uint32_t)(fminf(fmaxf(v, 0.0f), 1.0f) * 1023.0f);
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    return (x | (x << 2)) & 0x09249249u;
}

__device__ __forceinline__ uint32_t morton3(float ux, float uy, float uz) {
    return (spread(ux) << 2) | (spread(uy) << 1) | spread(uz);
}

// ---- scene box ----

__device__ __forceinline__ void warp_minmax(float* v) {
    for (int o = 16; o > 0; o >>= 1) {
        for (int k = 0; k < 3; k++) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
        for (int k = 3; k < 6; k++) v[k] = fmaxf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    }
}

// Reduces six values (3 min, 3 max) over a 256-thread block into s[0..6).
__device__ void block_minmax(float* v, float* s) {
    __shared__ float part[WARPS][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    warp_minmax(v);
    if (lane == 0)
        for (int k = 0; k < 6; k++) part[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < 6; k++) v[k] = lane < WARPS ? part[lane][k] : (k < 3 ? FLT_MAX : -FLT_MAX);
        warp_minmax(v);
        if (lane == 0)
            for (int k = 0; k < 6; k++) s[k] = v[k];
    }
    __syncthreads();
}

// Zeroes `words` words (the gated stand-in for a memset node).
__global__ void k_fill(uint32_t* __restrict__ p, size_t words, Gate gate) {
    if (gate.off()) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0u;
}

__global__ void __launch_bounds__(256) k_bounds(const float4* __restrict__ prims, uint32_t n, float4* __restrict__ partial,
                                                  Gate gate) {
    if (gate.off()) return;
    __shared__ float s[6];
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = __ldg(prims + 2 * (size_t)i), b = __ldg(prims + 2 * (size_t)i + 1);
        v[0] = fminf(v[0], a.x);
        v[1] = fminf(v[1], a.y);
        v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x);
        v[4] = fmaxf(v[4], b.y);
        v[5] = fmaxf(v[5], b.z);
    }
    block_minmax(v, s);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = make_float4(s[0], s[1], s[2], 0.0f);
        partial[2 * blockIdx.x + 1] = make_float4(s[3], s[4], s[5], 0.0f);
    }
}

// Finishes the scene box from the partials, then codes[i] (build.rs:75-85)
// and the four digit histograms of the sort.
__global__ void __launch_bounds__(256) k_morton_hist(const float4* __restrict__ prims, uint32_t n,
                                                     const float4* __restrict__ partial, uint32_t nparts,
                                                     uint32_t* __restrict__ codes, uint32_t* __restrict__ hist,
                                                     float4* __restrict__ scene_out, Gate gate) {
    if (gate.off()) return;
    __shared__ float s[6];
    __shared__ uint32_t s_hist[PASSES * 256];
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t k = threadIdx.x; k < nparts; k += blockDim.x) {
        const float4 a = partial[2 * k], b = partial[2 * k + 1];
        v[0] = fminf(v[0], a.x);
        v[1] = fminf(v[1], a.y);
        v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x);
        v[4] = fmaxf(v[4], b.y);
        v[5] = fmaxf(v[5], b.z);
    }
    for (int k = threadIdx.x; k < PASSES * 256; k += blockDim.x) s_hist[k] = 0;
    block_minmax(v, s);
    const float lo0 = s[0], lo1 = s[1], lo2 = s[2];
    const float e0 = s[3] - s[0], e1 = s[4] - s[1], e2 = s[5] - s[2];
    const float inv0 = e0 > 0.0f ? 1.0f / e0 : 0.0f;
    const float inv1 = e1 > 0.0f ? 1.0f / e1 : 0.0f;
    const float inv2 = e2 > 0.0f ? 1.0f / e2 : 0.0f;
    if (blockIdx.x == 0 && threadIdx.x == 0 && scene_out) {
        scene_out[0] = make_float4(s[0], s[1], s[2], 0.0f);
        scene_out[1] = make_float4(s[3], s[4], s[5], 0.0f);
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = __ldg(prims + 2 * (size_t)i), b = __ldg(prims + 2 * (size_t)i + 1);
        const float cx = 0.5f * (a.x + b.x), cy = 0.5f * (a.y + b.y), cz = 0.5f * (a.z + b.z);
        const uint32_t c = morton3((cx - lo0) * inv0, (cy - lo1) * inv1, (cz - lo2) * inv2);
        codes[i] = c;
        atomicAdd(&s_hist[0 * 256 + (c & 255)], 1u);
        atomicAdd(&s_hist[1 * 256 + ((c >> 8) & 255)], 1u);
        atomicAdd(&s_hist[2 * 256 + ((c >> 16) & 255)], 1u);
        atomicAdd(&s_hist[3 * 256 + (c >> 24)], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < PASSES * 256; k += blockDim.x)
        if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

// The reference's WGSL Morton kernel (kernel.rs:21-51), box given: the
// Pass-replayable form.
__global__ void k_morton_given(const float4* __restrict__ prims, uint32_t n, phx_morton_param p,
                               uint32_t* __restrict__ codes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(prims + 2 * (size_t)i), b = __ldg(prims + 2 * (size_t)i + 1);
    const float cx = 0.5f * (a.x + b.x), cy = 0.5f * (a.y + b.y), cz = 0.5f * (a.z + b.z);
    codes[i] = morton3((cx - p.lo[0]) * p.inv[0], (cy - p.lo[1]) * p.inv[1], (cz - p.lo[2]) * p.inv[2]);
}

__global__ void k_hist(const uint32_t* __restrict__ codes, uint32_t n, uint32_t* __restrict__ hist, Gate gate) {
    if (gate.off()) return;
    __shared__ uint32_t s_hist[PASSES * 256];
    for (int k = threadIdx.x; k < PASSES * 256; k += blockDim.x) s_hist[k] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = codes[i];
        atomicAdd(&s_hist[0 * 256 + (c & 255)], 1u);
        atomicAdd(&s_hist[1 * 256 + ((c >> 8) & 255)], 1u);
        atomicAdd(&s_hist[2 * 256 + ((c >> 16) & 255)], 1u);
        atomicAdd(&s_hist[3 * 256 + (c >> 24)], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < PASSES * 256; k += blockDim.x)
        if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

// ---- stable onesweep radix pass ----

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_tmp /* WARPS */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_tmp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < WARPS ? s_tmp[lane] : 0;
        uint32_t wi = w;
        for (int o = 1; o < WARPS; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < WARPS) s_tmp[lane] = wi - w;
    }
    __syncthreads();
    const uint32_t r = s_tmp[warp] + inc - v;
    __syncthreads();
    return r;
}

// One LSD pass over digit `shift`. Tiles of 4096 keys are taken in launch
// order (an atomic ticket), each warp ranks its 512 keys in order with
// __match_any_sync, the tile's per-digit counts are published and the
// prefix over earlier tiles found by decoupled look-back, and keys are
// staged in shared memory by digit so the global writes come out in runs.
// FIRST: the values are the indices (no value input).
template <bool FIRST>
__global__ void __launch_bounds__(RADIX_THREADS) k_radix_pass(const uint32_t* __restrict__ keys_in,
                                                              const uint32_t* __restrict__ vals_in,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ vals_out, uint32_t n,
                                                              uint32_t shift, const uint32_t* __restrict__ hist,
                                                              uint32_t* lookback, uint32_t* ticket,
                                                              uint32_t* status, Gate gate) {
    if (gate.off()) return;
    __shared__ uint32_t s_warp[WARPS][256];
    __shared__ uint32_t s_keys[TILE];
    __shared__ uint32_t s_vals[TILE];
    __shared__ uint32_t s_tile_off[256];
    __shared__ uint32_t s_glob[256];
    __shared__ uint32_t s_tmp[WARPS];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(ticket, 1u);
    for (int k = tid; k < WARPS * 256; k += RADIX_THREADS) (&s_warp[0][0])[k] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * TILE;
    const uint32_t wbase = base + warp * (32 * RADIX_ITEMS);

    uint32_t key[RADIX_ITEMS], val[RADIX_ITEMS], rank[RADIX_ITEMS];
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        const uint32_t idx = wbase + j * 32 + lane;
        const bool ok = idx < n;
        key[j] = ok ? keys_in[idx] : 0u;
        val[j] = FIRST ? idx : (ok ? vals_in[idx] : 0u);
    }
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        const bool ok = (wbase + j * 32 + lane) < n;
        const uint32_t d = (key[j] >> shift) & 255u;
        const uint32_t peers = __match_any_sync(0xffffffffu, ok ? d : 256u + lane);
        const uint32_t before = ok ? s_warp[warp][d] : 0u;
        __syncwarp();
        if (ok && lane == 31 - __clz(peers)) s_warp[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[j] = before + __popc(peers & lt);
    }
    __syncthreads();

    // Thread d owns digit d: warp offsets, the tile's count, the look-back.
    const uint32_t d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < WARPS; w++) {
        const uint32_t c = s_warp[w][d];
        s_warp[w][d] = run;
        run += c;
    }
    uint32_t* mine = lookback + (size_t)tile * 256 + d;
    uint32_t prefix = 0;
    if (tile == 0) {
        st_relaxed(mine, FLAG_INC | run);
    } else {
        st_relaxed(mine, FLAG_AGG | run);
        prefix = lookback_prefix(lookback, tile, d, SPIN_LIMIT, status);
        st_relaxed(mine, FLAG_INC | ((prefix + run) & VALUE_MASK));
    }
    const uint32_t tile_off = block_exclusive_scan(run, s_tmp);
    const uint32_t gbase = block_exclusive_scan(hist[d], s_tmp);
    s_tile_off[d] = tile_off;
    s_glob[d] = gbase + prefix;
    __syncthreads();

#pragma unroll
    for (int j = 0; j < RADIX_ITEMS; j++) {
        if ((wbase + j * 32 + lane) < n) {
            const uint32_t dd = (key[j] >> shift) & 255u;
            const uint32_t pos = s_tile_off[dd] + s_warp[warp][dd] + rank[j];
            s_keys[pos] = key[j];
            s_vals[pos] = val[j];
        }
    }
    __syncthreads();
    const uint32_t count = n - base < (uint32_t)TILE ? n - base : (uint32_t)TILE;
#pragma unroll
    for (int k = 0; k < RADIX_ITEMS; k++) {
        const uint32_t i = tid + k * RADIX_THREADS;
        if (i < count) {
            const uint32_t kk = s_keys[i];
            const uint32_t dd = (kk >> shift) & 255u;
            const uint32_t out = s_glob[dd] + (i - s_tile_off[dd]);
            keys_out[out] = kk;
            vals_out[out] = s_vals[i];
        }
    }
}

// ---- Karras (build.rs:28-60, kernel.rs:65-117) ----

__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ codes, long long n, long long i, long long j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = __ldg(codes + i), b = __ldg(codes + j);
    if (a != b) return __clz(a ^ b);
    return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

__device__ __forceinline__ uint4 karras_link(const uint32_t* __restrict__ codes, long long n, long long i) {
    const long long d = (kdelta(codes, n, i, i + 1) - kdelta(codes, n, i, i - 1) > 0) ? 1 : -1;
    const int dmin = kdelta(codes, n, i, i - d);
    long long lmax = 2;
    while (kdelta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
    long long l = 0, t = lmax / 2;
    while (t >= 1) {
        if (kdelta(codes, n, i, i + (l + t) * d) > dmin) l += t;
        t /= 2;
    }
    const long long j = i + l * d;
    const int dnode = kdelta(codes, n, i, j);
    long long s = 0;
    t = l;
    for (;;) {
        t = (t + 1) >> 1;
        if (kdelta(codes, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const long long g = i + s * d + (d < 0 ? d : 0);
    const long long first = i < j ? i : j, last = i < j ? j : i;
    const long long left = (first == g) ? n - 1 + g : g;
    const long long right = (last == g + 1) ? n + g : g + 1;
    return make_uint4((uint32_t)left, (uint32_t)right, (uint32_t)first, (uint32_t)last);
}

__global__ void __launch_bounds__(256) k_karras(const uint32_t* __restrict__ codes, uint32_t n, uint4* __restrict__ links,
                                                uint32_t* __restrict__ parent, Gate gate) {
    if (gate.off()) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && parent) parent[0] = NONE;
    if (i + 1 >= n) return;
    const uint4 L = karras_link(codes, n, i);
    links[i] = L;
    if (parent) {
        parent[L.x] = i;
        parent[L.y] = i;
    }
}

// ---- depth of every inner node by pointer jumping ----

// anc[i] starts as i's parent (the root its own), dist[i] as 1 (the root 0);
// each round doubles the hops: dist[i] += dist[anc[i]], anc[i] = anc[anc[i]].
// After DEPTH_ROUNDS rounds a node within 2^DEPTH_ROUNDS = STACK hops of the
// root has anc 0 and dist its depth; any deeper node has anc != 0.
constexpr int DEPTH_ROUNDS = 5;
static_assert((1u << DEPTH_ROUNDS) == STACK, "the jumps cover the stack's depth");

__global__ void __launch_bounds__(256) k_depth_init(const uint32_t* __restrict__ parent, uint32_t ninner,
                                                    uint32_t* __restrict__ anc, uint32_t* __restrict__ dist,
                                                    Gate gate) {
    if (gate.off()) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninner) return;
    anc[i] = i == 0 ? 0u : __ldg(parent + i);
    dist[i] = i == 0 ? 0u : 1u;
}

__global__ void __launch_bounds__(256) k_depth_jump(const uint32_t* __restrict__ anc, const uint32_t* __restrict__ dist,
                                                    uint32_t ninner, uint32_t* __restrict__ anc_out,
                                                    uint32_t* __restrict__ dist_out, Gate gate) {
    if (gate.off()) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninner) return;
    const uint32_t a = __ldg(anc + i);
    dist_out[i] = __ldg(dist + i) + __ldg(dist + a);
    anc_out[i] = __ldg(anc + a);
}

// ---- pack + depth (Bvh::assemble without the DFS) ----

__global__ void __launch_bounds__(256) k_pack(const uint4* __restrict__ links, const uint32_t* __restrict__ parent,
                                              const uint32_t* __restrict__ anc, const uint32_t* __restrict__ dist,
                                              uint32_t n, uint32_t leaf, float4* __restrict__ nodes,
                                              uint32_t* __restrict__ starts, uint32_t* __restrict__ nstarts,
                                              uint32_t* __restrict__ depth_out, Gate gate) {
    if (gate.off()) return;
    const uint32_t total = 2 * n - 1;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < total;
    bool reach = false, start = false;
    uint32_t dep = 0;
    if (active) {
        const bool internal = i + 1 < n;
        uint32_t lo_i, hi_i;
        uint4 L = make_uint4(0, 0, 0, 0);
        if (internal) {
            L = __ldg(links + i);
            lo_i = L.x;
            hi_i = L.y;
        } else {
            const uint32_t k = i - (n - 1);
            lo_i = k | LEAF;
            hi_i = k + 1;
        }
        if (i == 0) {
            reach = true;
        } else {
            const uint32_t p = __ldg(parent + i);
            const uint4 Lp = __ldg(links + p);
            if (Lp.w - Lp.z >= leaf) {
                // depth(p), or STACK for any depth past it (p is then cand
                // and i unreachable)
                const uint32_t dp = __ldg(anc + p) == 0 ? __ldg(dist + p) : STACK;
                if (dp + 1 < STACK) {
                    reach = true;
                    dep = dp + 1;
                }
            }
        }
        if (reach) {
            if (internal) {
                if (L.w - L.z < leaf || dep + 1 >= STACK) {
                    lo_i = L.z | LEAF;
                    hi_i = L.w + 1;
                    start = true;
                }
            } else {
                start = true;
            }
        }
        nodes[2 * (size_t)i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(lo_i));
        nodes[2 * (size_t)i + 1] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(hi_i));
    }
    // One atomic a block for the depth and one for the start list (a warp's
    // atomics on the two words serialised the kernel).
    __shared__ uint32_t s_max[8], s_cnt[8], s_base;
    const uint32_t dmax = __reduce_max_sync(0xffffffffu, reach ? dep : 0u);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t m = __ballot_sync(0xffffffffu, start);
    if (lane == 0) {
        s_max[warp] = dmax;
        s_cnt[warp] = __popc(m);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bm = 0, total = 0;
        for (int k = 0; k < 8; k++) {
            bm = bm > s_max[k] ? bm : s_max[k];
            const uint32_t c = s_cnt[k];
            s_cnt[k] = total;
            total += c;
        }
        if (bm) atomicMax(depth_out, bm);
        s_base = total ? atomicAdd(nstarts, total) : 0u;
    }
    __syncthreads();
    if (start) starts[s_base + s_cnt[warp] + __popc(m & ((1u << lane) - 1u))] = i;
}

// ---- refit: atomic bottom-up (Bvh::refit's bounds, Warp's refit pattern) ----

// `order` NULL: boxes are given by sorted slot (Bvh::refit_slots,
// build.rs:172-177). counters[] start even; each reachable inner node gets
// exactly two arrivals per refit, so no reset is needed between refits.
__global__ void __launch_bounds__(256) k_refit(const float4* __restrict__ prims, const uint32_t* __restrict__ order,
                                               const uint32_t* __restrict__ parent, float4* nodes,
                                               const uint32_t* __restrict__ starts,
                                               const uint32_t* __restrict__ nstarts, uint32_t* counters,
                                               uint32_t* status, Gate gate) {
    if (gate.off()) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nstarts) return;
    uint32_t i = starts[t];
    const float4 a = nodes[2 * (size_t)i], b = nodes[2 * (size_t)i + 1];
    const uint32_t first = __float_as_uint(a.w) & ~LEAF, end = __float_as_uint(b.w);
    float lx = FLT_MAX, ly = FLT_MAX, lz = FLT_MAX, hx = -FLT_MAX, hy = -FLT_MAX, hz = -FLT_MAX;
    for (uint32_t s = first; s < end; s++) {
        const uint32_t p = order ? __ldg(order + s) : s;
        const float4 pa = __ldg(prims + 2 * (size_t)p), pb = __ldg(prims + 2 * (size_t)p + 1);
        lx = fminf(lx, pa.x);
        ly = fminf(ly, pa.y);
        lz = fminf(lz, pa.z);
        hx = fmaxf(hx, pb.x);
        hy = fmaxf(hy, pb.y);
        hz = fmaxf(hz, pb.z);
    }
    nodes[2 * (size_t)i] = make_float4(lx, ly, lz, a.w);
    nodes[2 * (size_t)i + 1] = make_float4(hx, hy, hz, b.w);
    refit_climb(i, lx, ly, lz, hx, hy, hz, parent, nodes, counters, status);
}

// The reference's Jacobi Refit step (kernel.rs:130-170), for Pass replay.
__global__ void k_refit_jacobi(const float4* __restrict__ prims, const uint32_t* __restrict__ order,
                               const float4* __restrict__ src, float4* __restrict__ dst, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 a = src[2 * (size_t)k], b = src[2 * (size_t)k + 1];
    const uint32_t li = __float_as_uint(a.w), ri = __float_as_uint(b.w);
    float lx = 3.4028235e38f, ly = 3.4028235e38f, lz = 3.4028235e38f;
    float hx = -3.4028235e38f, hy = -3.4028235e38f, hz = -3.4028235e38f;
    if (li & LEAF) {
        for (uint32_t s = li & ~LEAF; s < ri; s++) {
            const uint32_t p = order[s];
            const float4 pa = prims[2 * (size_t)p], pb = prims[2 * (size_t)p + 1];
            lx = fminf(lx, pa.x);
            ly = fminf(ly, pa.y);
            lz = fminf(lz, pa.z);
            hx = fmaxf(hx, pb.x);
            hy = fmaxf(hy, pb.y);
            hz = fmaxf(hz, pb.z);
        }
    } else {
        const float4 la = src[2 * (size_t)li], lb = src[2 * (size_t)li + 1];
        const float4 ra = src[2 * (size_t)ri], rb = src[2 * (size_t)ri + 1];
        lx = fminf(la.x, ra.x);
        ly = fminf(la.y, ra.y);
        lz = fminf(la.z, ra.z);
        hx = fmaxf(lb.x, rb.x);
        hy = fmaxf(lb.y, rb.y);
        hz = fmaxf(lb.z, rb.z);
    }
    dst[2 * (size_t)k] = make_float4(lx, ly, lz, a.w);
    dst[2 * (size_t)k + 1] = make_float4(hx, hy, hz, b.w);
}

uint32_t grid_for(uint64_t items, uint32_t block, uint32_t cap) {
    uint64_t g = (items + block - 1) / block;
    if (g == 0) g = 1;
    return (uint32_t)(g < cap ? g : cap);
}

}  // namespace

int32_t BvhWork::reserve(uint32_t n, int sms) {
    if (n <= cap && prims.ptr) return PHX_OK;
    const size_t m = n ? n : 1;
    tiles = (uint32_t)((m + TILE - 1) / TILE);
    nparts = grid_for(m, 256, (uint32_t)sms * 4);
    PHX_TRY(prims.reserve(m * sizeof(phx_aabb)));
    PHX_TRY(codes.reserve(m * 4));
    PHX_TRY(sorted.reserve(m * 4));
    PHX_TRY(order.reserve(m * 4));
    PHX_TRY(alt_keys.reserve(m * 4));
    PHX_TRY(alt_vals.reserve(m * 4));
    PHX_TRY(partial.reserve((size_t)nparts * 32));
    PHX_TRY(zeroed.reserve(zeroed_bytes()));
    PHX_TRY(links.reserve(m * sizeof(phx_link)));
    PHX_TRY(parent.reserve((2 * m) * 4));
    PHX_TRY(nodes.reserve((2 * m) * sizeof(phx_node)));
    PHX_TRY(starts.reserve(m * 4));
    PHX_TRY(counters.reserve(m * 4));
    PHX_TRY(scalars.reserve(64));
    PHX_TRY(scene.reserve(sizeof(phx_aabb)));
    cap = (uint32_t)m;
    return PHX_OK;
}

// Zeroes `bytes` (a multiple of 4) on the stream: a memset node, or under a
// gate a kernel that reads the gate first.
static int32_t zero(Ctx* c, void* p, size_t bytes, Gate gate) {
    if (!gate.word) return cuda_check(cudaMemsetAsync(p, 0, bytes, c->stream), "memset");
    const size_t words = bytes / 4;
    k_fill<<<grid_for(words, 256, (uint32_t)c->sms * 4), 256, 0, c->stream>>>((uint32_t*)p, words, gate);
    return cuda_check(cudaGetLastError(), "fill");
}

// Stable LSD sort of `codes` (n keys): sorted codes and order into `w`.
static int32_t enqueue_sort(Ctx* c, BvhWork& w, const uint32_t* codes, uint32_t n, bool hist_ready,
                            Gate gate = Gate{}) {
    cudaStream_t s = c->stream;
    uint32_t tiles = (n + TILE - 1) / TILE;
    if (!hist_ready) {
        PHX_TRY(zero(c, w.zeroed.ptr, w.zeroed_bytes(), gate));
        k_hist<<<grid_for(n, 256, (uint32_t)c->sms * 4), 256, 0, s>>>(codes, n, w.hist(), gate);
        PHX_CUDA(cudaGetLastError());
    }
    uint32_t* ak = (uint32_t*)w.alt_keys.ptr;
    uint32_t* av = (uint32_t*)w.alt_vals.ptr;
    uint32_t* sk = (uint32_t*)w.sorted.ptr;
    uint32_t* sv = (uint32_t*)w.order.ptr;
    k_radix_pass<true><<<tiles, RADIX_THREADS, 0, s>>>(codes, nullptr, ak, av, n, 0, w.hist() + 0 * 256,
                                                        w.lookback(0), w.tickets() + 0, c->status, gate);
    k_radix_pass<false><<<tiles, RADIX_THREADS, 0, s>>>(ak, av, sk, sv, n, 8, w.hist() + 1 * 256, w.lookback(1),
                                                         w.tickets() + 1, c->status, gate);
    k_radix_pass<false><<<tiles, RADIX_THREADS, 0, s>>>(sk, sv, ak, av, n, 16, w.hist() + 2 * 256, w.lookback(2),
                                                         w.tickets() + 2, c->status, gate);
    k_radix_pass<false><<<tiles, RADIX_THREADS, 0, s>>>(ak, av, sk, sv, n, 24, w.hist() + 3 * 256, w.lookback(3),
                                                         w.tickets() + 3, c->status, gate);
    return cuda_check(cudaGetLastError(), "radix sort");
}

// The stable sort over caller-provided arrays: alt_keys/alt_vals hold n
// words each, hist 4 x 256 words, tickets 4 words and the look-back
// 4 x `stride` x 256 words (stride >= ceil(n / 4096)); hist, tickets and the
// look-back must be zero on entry.
int32_t enqueue_sort_raw(Ctx* c, const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted,
                         uint32_t* alt_keys, uint32_t* alt_vals, uint32_t* hist, uint32_t* tickets, uint32_t* lookback,
                         uint32_t stride) {
    if (n == 0) return PHX_OK;
    cudaStream_t s = c->stream;
    const uint32_t tiles = (n + TILE - 1) / TILE;
    k_hist<<<grid_for(n, 256, (uint32_t)c->sms * 4), 256, 0, s>>>(codes, n, hist, Gate{});
    for (int pass = 0; pass < PASSES; pass++) {
        const uint32_t* kin = pass == 0 ? codes : (pass % 2 == 1 ? alt_keys : sorted);
        const uint32_t* vin = pass % 2 == 1 ? alt_vals : order;
        uint32_t* kout = pass % 2 == 0 ? alt_keys : sorted;
        uint32_t* vout = pass % 2 == 0 ? alt_vals : order;
        uint32_t* lb = lookback + (size_t)pass * stride * 256;
        if (pass == 0)
            k_radix_pass<true><<<tiles, RADIX_THREADS, 0, s>>>(kin, nullptr, kout, vout, n, 0, hist, lb, tickets,
                                                                c->status, Gate{});
        else
            k_radix_pass<false><<<tiles, RADIX_THREADS, 0, s>>>(kin, vin, kout, vout, n, 8 * pass, hist + 256 * pass,
                                                                 lb, tickets + pass, c->status, Gate{});
    }
    return cuda_check(cudaGetLastError(), "radix sort");
}

// Every stage of Bvh::build over w.prims[0..n) on the context's stream.
int32_t enqueue_build(Ctx* c, BvhWork& w, uint32_t n, uint32_t leaf, Gate gate, bool refit) {
    cudaStream_t s = c->stream;
    PHX_TRY(zero(c, w.scalars.ptr, 64, gate));
    if (n == 0) return PHX_OK;
    const float4* prims = (const float4*)w.prims.ptr;
    const uint32_t nparts = grid_for(n, 256, (uint32_t)c->sms * 4);
    k_bounds<<<nparts, 256, 0, s>>>(prims, n, (float4*)w.partial.ptr, gate);
    PHX_TRY(zero(c, w.zeroed.ptr, w.zeroed_bytes(), gate));
    k_morton_hist<<<grid_for(n, 256, (uint32_t)c->sms * 8), 256, 0, s>>>(
        prims, n, (const float4*)w.partial.ptr, nparts, (uint32_t*)w.codes.ptr, w.hist(), (float4*)w.scene.ptr, gate);
    PHX_CUDA(cudaGetLastError());
    PHX_TRY(enqueue_sort(c, w, (const uint32_t*)w.codes.ptr, n, true, gate));
    k_karras<<<grid_for(n, 256, 1u << 30), 256, 0, s>>>((const uint32_t*)w.sorted.ptr, n, (uint4*)w.links.ptr,
                                                        (uint32_t*)w.parent.ptr, gate);
    PHX_TRY(zero(c, w.counters.ptr, (size_t)n * 4, gate));
    // Inner nodes' depths (the unsorted codes and the sort's ping-pong
    // arrays are free now; the depth rounds end in alt_keys / alt_vals).
    uint32_t* anc_a = (uint32_t*)w.codes.ptr;
    uint32_t* dist_a = (uint32_t*)w.starts.ptr;
    uint32_t* anc_b = (uint32_t*)w.alt_keys.ptr;
    uint32_t* dist_b = (uint32_t*)w.alt_vals.ptr;
    const uint32_t ninner = n - 1;
    if (ninner) {
        k_depth_init<<<grid_for(ninner, 256, 1u << 30), 256, 0, s>>>((const uint32_t*)w.parent.ptr, ninner, anc_a,
                                                                    dist_a, gate);
        for (int r = 0; r < DEPTH_ROUNDS; r++) {
            k_depth_jump<<<grid_for(ninner, 256, 1u << 30), 256, 0, s>>>(anc_a, dist_a, ninner, anc_b, dist_b, gate);
            std::swap(anc_a, anc_b);
            std::swap(dist_a, dist_b);
        }
    }
    static_assert(DEPTH_ROUNDS % 2 == 1, "the last round writes alt_keys / alt_vals, not starts");
    k_pack<<<grid_for(2ull * n - 1, 256, 1u << 30), 256, 0, s>>>((const uint4*)w.links.ptr,
                                                                (const uint32_t*)w.parent.ptr, anc_a, dist_a, n, leaf,
                                                                (float4*)w.nodes.ptr, (uint32_t*)w.starts.ptr,
                                                                w.nstarts(), w.depth(), gate);
    if (!refit) return cuda_check(cudaGetLastError(), "bvh build");
    k_refit<<<grid_for(n, 256, 1u << 30), 256, 0, s>>>(prims, (const uint32_t*)w.order.ptr,
                                                       (const uint32_t*)w.parent.ptr, (float4*)w.nodes.ptr,
                                                       (const uint32_t*)w.starts.ptr, w.nstarts(),
                                                       (uint32_t*)w.counters.ptr, c->status, gate);
    return cuda_check(cudaGetLastError(), "bvh build");
}

int32_t enqueue_refit(Ctx* c, BvhWork& w, uint32_t n, bool slots, Gate gate) {
    if (n == 0) return PHX_OK;
    k_refit<<<grid_for(n, 256, 1u << 30), 256, 0, c->stream>>>(
        (const float4*)w.prims.ptr, slots ? nullptr : (const uint32_t*)w.order.ptr, (const uint32_t*)w.parent.ptr,
        (float4*)w.nodes.ptr, (const uint32_t*)w.starts.ptr, w.nstarts(), (uint32_t*)w.counters.ptr, c->status, gate);
    return cuda_check(cudaGetLastError(), "bvh refit");
}

int32_t launch_morton_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items) {
    phx_morton_param p;
    memcpy(&p, params, sizeof p);
    if (items == 0) return PHX_OK;
    const uint32_t n = items < p.n ? items : p.n;
    k_morton_given<<<grid_for(n, 256, 1u << 30), 256, 0, s>>>((const float4*)bufs[0], n, p, (uint32_t*)bufs[1]);
    return cuda_check(cudaGetLastError(), "morton");
}

int32_t launch_karras_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items) {
    phx_karras_param p;
    memcpy(&p, params, sizeof p);
    if (items == 0 || p.leaves < 2) return PHX_OK;
    k_karras<<<grid_for(items, 256, 1u << 30), 256, 0, s>>>((const uint32_t*)bufs[0], p.leaves, (uint4*)bufs[1],
                                                            nullptr, Gate{});
    return cuda_check(cudaGetLastError(), "karras");
}

int32_t launch_refit_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items) {
    phx_refit_param p;
    memcpy(&p, params, sizeof p);
    if (items == 0) return PHX_OK;
    const uint32_t n = items < p.n ? items : p.n;
    k_refit_jacobi<<<grid_for(n, 256, 1u << 30), 256, 0, s>>>((const float4*)bufs[0], (const uint32_t*)bufs[1],
                                                              (const float4*)bufs[2], (float4*)bufs[3], n);
    return cuda_check(cudaGetLastError(), "refit step");
}

}  // namespace phx

using namespace phx;

struct phx_bvh_s {
    Ctx* ctx = nullptr;
    uint32_t n = 0, leaf = 4;
    BvhWork w;
};

static int32_t bvh_new(phx_ctx ctx, uint32_t n, uint32_t leaf, phx_bvh* out) {
    if (!ctx || !out) return fail(PHX_ERR_INVALID, "null argument");
    if (n >= MAX_PRIMS) return fail(PHX_ERR_INVALID, "%u prims: at most 2^30 - 1", n);
    if (leaf == 0) return fail(PHX_ERR_INVALID, "leaf size 0");
    PHX_TRY(use(&ctx->c));
    auto* b = new phx_bvh_s();
    b->ctx = &ctx->c;
    b->n = n;
    b->leaf = leaf;
    int32_t rc = b->w.reserve(n, ctx->c.sms);
    if (rc != PHX_OK) {
        delete b;
        return rc;
    }
    ctx->c.live++;
    *out = b;
    return PHX_OK;
}

extern "C" {

int32_t phx_bvh_build(phx_ctx ctx, const phx_aabb* host_prims, uint32_t n, uint32_t leaf, phx_bvh* out) {
    if (n && !host_prims) return fail(PHX_ERR_INVALID, "null prims");
    phx_bvh b = nullptr;
    PHX_TRY(bvh_new(ctx, n, leaf, &b));
    int32_t rc = PHX_OK;
    if (n) rc = cuda_check(cudaMemcpyAsync(b->w.prims.ptr, host_prims, (size_t)n * sizeof(phx_aabb),
                                           cudaMemcpyHostToDevice, b->ctx->stream),
                           "upload prims");
    if (rc == PHX_OK) rc = enqueue_build(b->ctx, b->w, n, leaf);
    // The host array is the caller's again on return.
    if (rc == PHX_OK) rc = wait_stream(b->ctx->stream, 0);
    if (rc != PHX_OK) {
        phx_bvh_destroy(b);
        return rc;
    }
    *out = b;
    return PHX_OK;
}

int32_t phx_bvh_build_device(phx_ctx ctx, const phx_aabb* device_prims, uint32_t n, uint32_t leaf, phx_bvh* out) {
    if (n && !device_prims) return fail(PHX_ERR_INVALID, "null prims");
    phx_bvh b = nullptr;
    PHX_TRY(bvh_new(ctx, n, leaf, &b));
    int32_t rc = PHX_OK;
    if (n) rc = cuda_check(cudaMemcpyAsync(b->w.prims.ptr, device_prims, (size_t)n * sizeof(phx_aabb),
                                           cudaMemcpyDeviceToDevice, b->ctx->stream),
                           "copy prims");
    if (rc == PHX_OK) rc = enqueue_build(b->ctx, b->w, n, leaf);
    if (rc != PHX_OK) {
        phx_bvh_destroy(b);
        return rc;
    }
    *out = b;
    return PHX_OK;
}

int32_t phx_bvh_rebuild_device(phx_bvh bvh, const phx_aabb* device_prims, uint32_t n) {
    if (!bvh || (n && !device_prims)) return fail(PHX_ERR_INVALID, "null argument");
    if (n >= MAX_PRIMS) return fail(PHX_ERR_INVALID, "%u prims: at most 2^30 - 1", n);
    PHX_TRY(use(bvh->ctx));
    if (n > bvh->w.cap) {
        PHX_TRY(wait_stream(bvh->ctx->stream, 0));
        PHX_TRY(bvh->w.reserve(n, bvh->ctx->sms));
    }
    bvh->n = n;
    if (n && (const void*)device_prims != bvh->w.prims.ptr)
        PHX_CUDA(cudaMemcpyAsync(bvh->w.prims.ptr, device_prims, (size_t)n * sizeof(phx_aabb),
                                 cudaMemcpyDeviceToDevice, bvh->ctx->stream));
    return enqueue_build(bvh->ctx, bvh->w, n, bvh->leaf);
}

int32_t phx_bvh_refit(phx_bvh bvh) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    PHX_TRY(use(bvh->ctx));
    return enqueue_refit(bvh->ctx, bvh->w, bvh->n, false);
}

int32_t phx_bvh_update(phx_bvh bvh, const phx_aabb* host_prims, uint32_t n) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    if (n != bvh->n) return PHX_REBUILD;
    if (n && !host_prims) return fail(PHX_ERR_INVALID, "null prims");
    PHX_TRY(use(bvh->ctx));
    if (n)
        PHX_CUDA(cudaMemcpyAsync(bvh->w.prims.ptr, host_prims, (size_t)n * sizeof(phx_aabb), cudaMemcpyHostToDevice,
                                 bvh->ctx->stream));
    PHX_TRY(enqueue_refit(bvh->ctx, bvh->w, n, false));
    return wait_stream(bvh->ctx->stream, 0);
}

int32_t phx_bvh_update_device(phx_bvh bvh, const phx_aabb* device_prims, uint32_t n) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    if (n != bvh->n) return PHX_REBUILD;
    if (n && !device_prims) return fail(PHX_ERR_INVALID, "null prims");
    PHX_TRY(use(bvh->ctx));
    if (n && (const void*)device_prims != bvh->w.prims.ptr)
        PHX_CUDA(cudaMemcpyAsync(bvh->w.prims.ptr, device_prims, (size_t)n * sizeof(phx_aabb),
                                 cudaMemcpyDeviceToDevice, bvh->ctx->stream));
    return enqueue_refit(bvh->ctx, bvh->w, n, false);
}

int32_t phx_bvh_download(phx_bvh bvh, phx_node* nodes, uint32_t* order, uint32_t* depth, uint32_t timeout_ms) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    PHX_TRY(use(bvh->ctx));
    cudaStream_t s = bvh->ctx->stream;
    const uint32_t n = bvh->n;
    if (nodes && n) PHX_CUDA(cudaMemcpyAsync(nodes, bvh->w.nodes.ptr, (2 * (size_t)n - 1) * sizeof(phx_node),
                                             cudaMemcpyDeviceToHost, s));
    if (order && n) PHX_CUDA(cudaMemcpyAsync(order, bvh->w.order.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    uint32_t d = 0;
    PHX_CUDA(cudaMemcpyAsync(&d, bvh->w.depth(), 4, cudaMemcpyDeviceToHost, s));
    PHX_TRY(wait_stream(s, timeout_ms));
    if (depth) *depth = d;
    return read_status(bvh->ctx);
}

int32_t phx_bvh_info(phx_bvh bvh, uint32_t* n, uint32_t* nodes, uint32_t* leaf, uint32_t* depth) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    if (n) *n = bvh->n;
    if (nodes) *nodes = bvh->n ? 2 * bvh->n - 1 : 0;
    if (leaf) *leaf = bvh->leaf;
    if (depth) {
        PHX_TRY(use(bvh->ctx));
        uint32_t d = 0;
        PHX_CUDA(cudaMemcpyAsync(&d, bvh->w.depth(), 4, cudaMemcpyDeviceToHost, bvh->ctx->stream));
        PHX_TRY(wait_stream(bvh->ctx->stream, 0));
        *depth = d;
    }
    return PHX_OK;
}

int32_t phx_bvh_device(phx_bvh bvh, phx_aabb** prims, uint32_t** order, phx_node** nodes, uint32_t** codes) {
    if (!bvh) return fail(PHX_ERR_INVALID, "null bvh");
    if (prims) *prims = (phx_aabb*)bvh->w.prims.ptr;
    if (order) *order = (uint32_t*)bvh->w.order.ptr;
    if (nodes) *nodes = (phx_node*)bvh->w.nodes.ptr;
    if (codes) *codes = (uint32_t*)bvh->w.sorted.ptr;
    return PHX_OK;
}

int32_t phx_bvh_destroy(phx_bvh bvh) {
    if (!bvh) return PHX_OK;
    use(bvh->ctx);
    cudaStreamSynchronize(bvh->ctx->stream);
    bvh->ctx->live--;
    delete bvh;
    return PHX_OK;
}

int32_t phx_morton(phx_ctx ctx, const phx_aabb* prims, uint32_t n, uint32_t* codes, phx_aabb* scene_out) {
    if (!ctx || (n && (!prims || !codes))) return fail(PHX_ERR_INVALID, "null argument");
    if (n == 0) return PHX_OK;
    Ctx* c = &ctx->c;
    PHX_TRY(use(c));
    DevMem partial, hist, scene;
    const uint32_t nparts = grid_for(n, 256, (uint32_t)c->sms * 4);
    PHX_TRY(partial.reserve((size_t)nparts * 32));
    PHX_TRY(hist.reserve(PASSES * 256 * 4));
    PHX_TRY(scene.reserve(32));
    PHX_CUDA(cudaMemsetAsync(hist.ptr, 0, PASSES * 256 * 4, c->stream));
    k_bounds<<<nparts, 256, 0, c->stream>>>((const float4*)prims, n, (float4*)partial.ptr, Gate{});
    k_morton_hist<<<grid_for(n, 256, (uint32_t)c->sms * 8), 256, 0, c->stream>>>(
        (const float4*)prims, n, (const float4*)partial.ptr, nparts, codes, (uint32_t*)hist.ptr,
        (float4*)(scene_out ? (void*)scene_out : scene.ptr), Gate{});
    PHX_CUDA(cudaGetLastError());
    return wait_stream(c->stream, 0);
}

int32_t phx_sort_codes(phx_ctx ctx, const uint32_t* codes, uint32_t n, uint32_t* order, uint32_t* sorted) {
    if (!ctx || (n && (!codes || !order || !sorted))) return fail(PHX_ERR_INVALID, "null argument");
    if (n >= MAX_PRIMS) return fail(PHX_ERR_INVALID, "%u keys: at most 2^30 - 1", n);
    if (n == 0) return PHX_OK;
    Ctx* c = &ctx->c;
    PHX_TRY(use(c));
    BvhWork w;
    PHX_TRY(w.reserve(n, c->sms));
    PHX_TRY(enqueue_sort(c, w, codes, n, false));
    PHX_CUDA(cudaMemcpyAsync(order, w.order.ptr, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->stream));
    PHX_CUDA(cudaMemcpyAsync(sorted, w.sorted.ptr, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->stream));
    PHX_TRY(wait_stream(c->stream, 0));
    return read_status(c);
}

int32_t phx_karras(phx_ctx ctx, const uint32_t* sorted, uint32_t n, phx_link* links) {
    if (!ctx || (n > 1 && (!sorted || !links))) return fail(PHX_ERR_INVALID, "null argument");
    if (n < 2) return PHX_OK;
    Ctx* c = &ctx->c;
    PHX_TRY(use(c));
    k_karras<<<grid_for(n, 256, 1u << 30), 256, 0, c->stream>>>(sorted, n, (uint4*)links, nullptr, Gate{});
    PHX_CUDA(cudaGetLastError());
    return wait_stream(c->stream, 0);
}

}  // extern "C"
