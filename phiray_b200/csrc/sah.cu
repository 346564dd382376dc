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
// One thread per node keeps the per-node arithmetic the reference's,
// but the top levels run on a handful of threads; splitting those nodes
// over whole blocks is the next step for speed.
#include "internal.cuh"
#include "sah_core.cuh"

namespace phx {
namespace {

using sah::TNode;

__device__ uint32_t atomic_add(uint32_t* p, uint32_t v) { return atomicAdd(p, v); }

struct DeviceAdd {
    __device__ uint32_t operator()(uint32_t* p, uint32_t v) const { return atomic_add(p, v); }
};

__global__ void k_sah_init(const float* __restrict__ prims, uint32_t n, float* __restrict__ centres,
                           uint32_t* __restrict__ order) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // Aabb::center (node.rs:90-92)
    for (int k = 0; k < 3; k++) centres[3 * (uint64_t)i + k] = 0.5f * (prims[8 * (uint64_t)i + k] + prims[8 * (uint64_t)i + 4 + k]);
    order[i] = i;
}

__global__ void k_sah_level(const uint32_t* __restrict__ list, uint32_t count, TNode* tn, const float* __restrict__ prims,
                            const float* __restrict__ centres, uint32_t* order, uint32_t leaf, uint32_t* tcount,
                            uint32_t* next, uint32_t* next_count) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    sah::process(list[k], tn, prims, centres, order, leaf, tcount, next, next_count, DeviceAdd{});
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
    std::vector<uint32_t> off{0}, len{1};
    for (uint32_t lv = 0; lv < sah::MAX_DEPTH; lv++) {
        const uint32_t next = off[lv] + len[lv];
        PHX_CUDA(cudaMemsetAsync(cnt + 1, 0, 4, s));
        k_sah_level<<<blocks_of(len[lv], 64), 64, 0, s>>>(L + off[lv], len[lv], T, P, (const float*)centres.ptr, order,
                                                         leaf, cnt, L + next, cnt + 1);
        PHX_CUDA(cudaGetLastError());
        uint32_t opened = 0;
        PHX_CUDA(cudaMemcpyAsync(&opened, cnt + 1, 4, cudaMemcpyDeviceToHost, s));
        PHX_TRY(wait_stream(s, 0));
        if (opened == 0) break;
        if (next + opened > cap) return fail(PHX_ERR_DEVICE, "SAH build: more nodes than 2n - 1");
        off.push_back(next);
        len.push_back(opened);
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
