// phx_selftest_wait: the library's bounded device waits, made to run out.
//
// Every wait in these kernels on something another thread or block must
// produce — an mbarrier phase the tensor-core engine commits to, a radix-sort
// tile's look-back word — polls at most a fixed number of times and then sets
// STATUS_SPIN_LIMIT in the context's status word and returns, so a lost
// producer costs an error code, not a hung GPU. This entry point runs those
// same wait helpers on a flag nothing sets (or, `satisfied`, on one that is
// already set), with a caller-chosen short limit, so a test can watch the
// wait give up and the host report it while the context stays usable.
#include "lbvh.cuh"
#include "tc.cuh"

namespace phx {
namespace {

// mbarrier: one thread waits for phase 0 of a barrier expecting one arrival,
// which it makes first only when `satisfied`.
__global__ void k_wait_mbarrier(uint32_t limit, int satisfied, uint32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (satisfied) tc::mbar_arrive(&bar);
        if (!tc::mbar_wait(&bar, 0, limit)) atomicOr(status, STATUS_SPIN_LIMIT);
    }
}

// look-back: the 256 digit threads of tile 1 wait for tile 0's words, which
// hold an inclusive prefix only when `satisfied` (else zero: not written).
__global__ void k_wait_lookback(uint32_t* words, uint32_t limit, uint32_t* status, uint32_t* out) {
    const uint32_t d = threadIdx.x;
    out[d] = lookback_prefix(words, 1, d, limit, status);
}

}  // namespace
}  // namespace phx

extern "C" int32_t phx_selftest_wait(phx_ctx ctx, int32_t which, uint32_t limit, int32_t satisfied) {
    using namespace phx;
    if (!ctx || (which != 0 && which != 1) || limit == 0) return fail(PHX_ERR_INVALID, "bad argument");
    Ctx* c = &ctx->c;
    PHX_TRY(use(c));
    if (which == 0) {
        k_wait_mbarrier<<<1, 32, 0, c->stream>>>(limit, satisfied, c->status);
        PHX_CUDA(cudaGetLastError());
    } else {
        void* p = nullptr;
        PHX_TRY(ctx_alloc(c, &p, 2 * 256 * 4 + 256 * 4));
        uint32_t* words = (uint32_t*)p;
        PHX_CUDA(cudaMemsetAsync(words, 0, 2 * 256 * 4, c->stream));
        if (satisfied) {
            std::vector<uint32_t> inc(256, LOOKBACK_INC | 7u);
            PHX_CUDA(cudaMemcpyAsync(words, inc.data(), 256 * 4, cudaMemcpyHostToDevice, c->stream));
        }
        k_wait_lookback<<<1, 256, 0, c->stream>>>(words, limit, c->status, words + 512);
        const cudaError_t e = cudaGetLastError();
        PHX_TRY(wait_stream(c->stream, 0));
        ctx_free(c, p);
        PHX_CUDA(e);
    }
    PHX_TRY(wait_stream(c->stream, 0));
    return read_status(c);
}
