// Internal declarations shared by the phiray-b200 CUDA sources: the context,
// buffers, error reporting and the device helpers every kernel file uses.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <string>
#include <vector>

#include "../../include/phiray_cuda.h"

namespace phx {

// Status word bits a kernel sets instead of trapping (read on the host at the
// next wait): a bounded spin ran out, or an input index was out of range.
enum : uint32_t {
    STATUS_SPIN_LIMIT = 1u << 0,
    STATUS_BAD_INDEX = 1u << 1,
    STATUS_STACK_OVERFLOW = 1u << 2,
};

struct Ctx;

// A growable device allocation. Reserved inside a context's call (after
// use()), it comes from the context's stream-ordered pool on the context's
// stream, and its release is a free ordered on that stream: the pool keeps
// the memory mapped, so the next object of the context reuses it without a
// cudaMalloc/cudaFree round trip through the driver. Otherwise cudaMalloc.
struct DevMem {
    void* ptr = nullptr;
    size_t bytes = 0;
    Ctx* owner = nullptr;          // the context whose pool holds ptr, or null
    int32_t reserve(size_t want);  // grows, discarding contents
    void release();
    ~DevMem() { release(); }
};

struct Ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t own = nullptr;     // created by phx_ctx_create
    cudaStream_t stream = nullptr;  // where work goes (own, or a caller's)
    cudaStream_t capture = nullptr; // private stream for graph capture
    uint32_t* status = nullptr;     // device status word
    cudaMemPool_t pool = nullptr;   // device memory of the context's objects
    DevMem denoise_scratch;         // guide and ping-pong planes of phx_denoise
    int live = 0;                   // buffers, passes, BVHs, tracers not yet freed
};

// Sets the thread's last error text and returns `code`.
int32_t fail(int32_t code, const char* fmt, ...);
// Maps a CUDA error to PHX_ERR_*, with context text; PHX_OK on success.
int32_t cuda_check(cudaError_t e, const char* what);
// Reads and clears the context's status word (synchronous), mapping set bits
// to PHX_ERR_KERNEL.
int32_t read_status(Ctx* c);
// Bounded drain of `stream` (polls an event with a deadline).
int32_t wait_stream(cudaStream_t s, uint32_t timeout_ms);
// Ensures ctx's device is current on this thread and makes ctx the one whose
// pool this thread's DevMem reservations draw on.
int32_t use(Ctx* c);
// Device allocation from the context's pool, ordered on its stream (cudaMalloc
// when the context has no pool); the matching free.
int32_t ctx_alloc(Ctx* c, void** p, size_t bytes);
void ctx_free(Ctx* c, void* p);

// Kernel launches the Pass layer replays (one per phx_kernel_id), defined in
// the kernel files. `params` is the step's params blob, `bufs` its buffers.
int32_t launch_skin_step(cudaStream_t s, const void* params, void* const* bufs, const uint64_t* sizes, uint32_t items,
                         uint32_t* status);
int32_t launch_denoise_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items);
int32_t launch_morton_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items);
int32_t launch_karras_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items);
int32_t launch_refit_step(cudaStream_t s, const void* params, void* const* bufs, uint32_t items);

// Face boxes (Aabb::of_tri) of vec4 vertices over uvec4 faces (skin.cu).
int32_t launch_face_boxes(cudaStream_t s, const float* verts, const uint32_t* faces, uint32_t nfaces, phx_aabb* boxes);

inline uint32_t ceil_div(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace phx

struct phx_ctx_s {
    phx::Ctx c;
};

struct phx_buf_s {
    phx::Ctx* ctx = nullptr;
    void* ptr = nullptr;
    uint64_t bytes = 0;
    bool owned = false;
};

#define PHX_TRY(expr)                   \
    do {                                \
        int32_t _rc = (expr);           \
        if (_rc < 0) return _rc;        \
    } while (0)

#define PHX_CUDA(expr) PHX_TRY(phx::cuda_check((expr), #expr))
