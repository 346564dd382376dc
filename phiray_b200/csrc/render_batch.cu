// The batched persistent launch (many tracers' frames in one launch) at its
// three block sizes and two register budgets, single-instance and full mode.
#include "render.cuh"

namespace phx {
namespace {

template <int THREADS, int M, int RES>
int32_t launch_batch_mode(bool smem_stack, int device, int sms, const void* jobs, uint32_t njobs, uint32_t ntiles,
                          uint32_t* next, cudaStream_t s) {
    const void* fn = (const void*)k_render_batch<M, THREADS, RES>;
    const int smem = smem_stack ? STACK * 4 * THREADS : 0;
    static std::atomic<uint64_t> done{0};  // per kernel form (one static a template instance)
    const uint64_t bit = 1ull << (device & 63);
    if (smem && !(done.load() & bit)) {
        PHX_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, STACK * 4 * THREADS));
        done.fetch_or(bit);
    }
    int per_sm = 0;
    PHX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, THREADS, smem));
    uint32_t grid = (uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sms;
    grid = std::min<uint32_t>(grid, (ntiles + THREADS / 32 - 1) / (THREADS / 32));
    if (grid == 0) return PHX_OK;
    PHX_CUDA(cudaMemsetAsync(next, 0, 4, s));
    k_render_batch<M, THREADS, RES><<<grid, THREADS, smem, s>>>((const Job*)jobs, njobs, ntiles, next);
    return cuda_check(cudaGetLastError(), "batch render");
}

template <int THREADS>
int32_t launch_batch_threads(bool full, bool smem_stack, bool dense, int device, int sms, const void* jobs,
                             uint32_t njobs, uint32_t ntiles, uint32_t* next, cudaStream_t s) {
    if (dense) {
        if (full)
            return launch_batch_mode<THREADS, MODE_FULL, 2048>(smem_stack, device, sms, jobs, njobs, ntiles, next, s);
        return launch_batch_mode<THREADS, 0, 2048>(smem_stack, device, sms, jobs, njobs, ntiles, next, s);
    }
    if (full) return launch_batch_mode<THREADS, MODE_FULL, 1536>(smem_stack, device, sms, jobs, njobs, ntiles, next, s);
    return launch_batch_mode<THREADS, 0, 1536>(smem_stack, device, sms, jobs, njobs, ntiles, next, s);
}

}  // namespace

size_t batch_job_bytes() { return sizeof(Job); }

int32_t render_batch(int threads, bool full, bool smem_stack, bool dense, int device, int sms, const void* jobs,
                     uint32_t njobs, uint32_t ntiles, uint32_t* next, cudaStream_t s) {
    switch (threads) {
        case 64: return launch_batch_threads<64>(full, smem_stack, dense, device, sms, jobs, njobs, ntiles, next, s);
        case 256: return launch_batch_threads<256>(full, smem_stack, dense, device, sms, jobs, njobs, ntiles, next, s);
        default: return launch_batch_threads<128>(full, smem_stack, dense, device, sms, jobs, njobs, ntiles, next, s);
    }
}

}  // namespace phx
