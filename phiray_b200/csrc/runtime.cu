// The runtime under the C ABI: context (phiray Gpu), buffers (GpuArray) and
// recorded passes (Pass) replayed as CUDA graphs.
//
// Reference: src/gpu/mod.rs (Gpu, wait_for, patience), src/gpu/array.rs
// (GpuArray), src/gpu/pass.rs (Pass), src/kernel/mod.rs (Kernel, Dispatch).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <unordered_set>

#include "internal.cuh"

namespace phx {

static thread_local std::string g_last_error;
// The context of this thread's last use(): DevMem::reserve draws on its pool.
static thread_local Ctx* t_current = nullptr;
// Contexts not yet destroyed (a stale t_current is never dereferenced).
static std::mutex g_ctx_mutex;
static std::unordered_set<Ctx*> g_ctxs;

static bool ctx_alive(Ctx* c) {
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    return g_ctxs.count(c) != 0;
}

int32_t fail(int32_t code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int32_t cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PHX_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(PHX_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    }
    return fail(PHX_ERR_DEVICE, "%s: %s", what, cudaGetErrorString(e));
}

int32_t use(Ctx* c) {
    if (!c) return fail(PHX_ERR_INVALID, "null context");
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != c->device) PHX_CUDA(cudaSetDevice(c->device));
    t_current = c;
    return PHX_OK;
}

int32_t ctx_alloc(Ctx* c, void** p, size_t bytes) {
    *p = nullptr;
    if (!c->pool) return cuda_check(cudaMalloc(p, bytes), "cudaMalloc");
    // An allocation recorded into a graph would belong to the graph: refuse
    // one made while the context's stream is being captured.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PHX_CUDA(cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        return fail(PHX_ERR_INVALID, "allocation of %zu bytes while the stream is captured", bytes);
    PHX_CUDA(cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream));
    // Kernels stage rows with 16-byte copies and vector loads: keep the
    // 256-byte alignment cudaMalloc gives.
    if ((uintptr_t)*p & 255u) {
        cudaFreeAsync(*p, c->stream);
        *p = nullptr;
        return fail(PHX_ERR_DEVICE, "pool allocation of %zu bytes not 256-byte aligned", bytes);
    }
    return PHX_OK;
}

void ctx_free(Ctx* c, void* p) {
    if (!p) return;
    if (c && c->pool) cudaFreeAsync(p, c->stream);
    else cudaFree(p);
}

int32_t wait_stream(cudaStream_t s, uint32_t timeout_ms) {
    // Gpu::wait_for (mod.rs:292-303): a bounded wait. The stream is polled,
    // never blocked on, so a device that stops answering becomes
    // PHX_ERR_TIMEOUT instead of a hung caller.
    if (timeout_ms == 0) timeout_ms = PHX_DEFAULT_WAIT_MS;
    cudaEvent_t ev;
    PHX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, s);
    if (e != cudaSuccess) {
        cudaEventDestroy(ev);
        return cuda_check(e, "cudaEventRecord");
    }
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    int spins = 0;
    for (;;) {
        e = cudaEventQuery(ev);
        if (e != cudaErrorNotReady) break;
        if (std::chrono::steady_clock::now() > deadline) {
            cudaEventDestroy(ev);
            return fail(PHX_ERR_TIMEOUT, "device did not drain within %u ms", timeout_ms);
        }
        if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    cudaEventDestroy(ev);
    return cuda_check(e, "stream wait");
}

int32_t read_status(Ctx* c) {
    uint32_t st = 0;
    PHX_CUDA(cudaMemcpyAsync(&st, c->status, 4, cudaMemcpyDeviceToHost, c->stream));
    PHX_TRY(wait_stream(c->stream, 0));
    if (st != 0) {
        PHX_CUDA(cudaMemsetAsync(c->status, 0, 4, c->stream));
        return fail(PHX_ERR_KERNEL, "kernel status 0x%x (%s%s%s)", st, (st & STATUS_SPIN_LIMIT) ? "spin limit " : "",
                    (st & STATUS_BAD_INDEX) ? "index out of range " : "",
                    (st & STATUS_STACK_OVERFLOW) ? "stack overflow" : "");
    }
    return PHX_OK;
}

int32_t DevMem::reserve(size_t want) {
    if (want <= bytes && ptr) return PHX_OK;
    release();
    if (want == 0) return PHX_OK;
    Ctx* c = t_current;
    int cur = -1;
    if (c && ctx_alive(c) && cudaGetDevice(&cur) == cudaSuccess && cur == c->device) {
        PHX_TRY(ctx_alloc(c, &ptr, want));
        owner = c;
    } else {
        PHX_CUDA(cudaMalloc(&ptr, want));
    }
    bytes = want;
    return PHX_OK;
}

void DevMem::release() {
    if (ptr) ctx_free(owner, ptr);
    ptr = nullptr;
    bytes = 0;
    owner = nullptr;
}

}  // namespace phx

using namespace phx;

extern "C" {

const char* phx_version(void) { return "phiray-b200 0.1 (sm_100a)"; }

int32_t phx_last_error(char* buf, size_t len) {
    const std::string& s = g_last_error;
    if (buf && len) {
        size_t k = s.size() < len - 1 ? s.size() : len - 1;
        std::memcpy(buf, s.data(), k);
        buf[k] = 0;
    }
    return (int32_t)s.size();
}

int32_t phx_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int32_t phx_ctx_create(int32_t ordinal, phx_ctx* out) {
    if (!out) return fail(PHX_ERR_INVALID, "null out");
    *out = nullptr;
    int n = phx_device_count();
    if (n <= 0) return fail(PHX_ERR_DEVICE, "no CUDA device");
    if (ordinal < 0 || ordinal >= n) return fail(PHX_ERR_INVALID, "device %d of %d", ordinal, n);
    PHX_CUDA(cudaSetDevice(ordinal));
    auto* h = new phx_ctx_s();
    Ctx& c = h->c;
    c.device = ordinal;
    cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, ordinal);
    {
        std::lock_guard<std::mutex> lock(g_ctx_mutex);
        g_ctxs.insert(&c);
    }
    // The context's memory pool: freed blocks stay mapped (up to a quarter of
    // the device) for the context's next objects. Without stream-ordered
    // allocation support the context uses cudaMalloc.
    int pools = 0;
    cudaDeviceGetAttribute(&pools, cudaDevAttrMemoryPoolsSupported, ordinal);
    if (pools) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ordinal;
        if (cudaMemPoolCreate(&c.pool, &props) == cudaSuccess) {
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            uint64_t keep = total_b / 4;
            cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            cudaGetLastError();
            c.pool = nullptr;
        }
    }
    int32_t rc = cuda_check(cudaStreamCreateWithFlags(&c.own, cudaStreamNonBlocking), "stream");
    if (rc == PHX_OK) rc = cuda_check(cudaStreamCreateWithFlags(&c.capture, cudaStreamNonBlocking), "stream");
    if (rc == PHX_OK) rc = cuda_check(cudaMalloc(&c.status, 4), "status");
    if (rc == PHX_OK) rc = cuda_check(cudaMemset(c.status, 0, 4), "status");
    if (rc != PHX_OK) {
        phx_ctx_destroy(h);
        return rc;
    }
    c.stream = c.own;
    *out = h;
    return PHX_OK;
}

int32_t phx_ctx_destroy(phx_ctx ctx) {
    if (!ctx) return PHX_OK;
    Ctx& c = ctx->c;
    // Everything made on a context holds a pointer to it: refuse to free it
    // under them (the caller frees buffers, passes, BVHs, tracers first).
    if (c.live > 0) return fail(PHX_ERR_INVALID, "context still has %d live objects", c.live);
    cudaSetDevice(c.device);
    {
        std::lock_guard<std::mutex> lock(g_ctx_mutex);
        g_ctxs.erase(&c);
    }
    if (t_current == &c) t_current = nullptr;
    if (c.stream) c.denoise_scratch.release();
    if (c.stream) cudaStreamSynchronize(c.stream);
    if (c.own) cudaStreamSynchronize(c.own);
    if (c.status) cudaFree(c.status);
    if (c.capture) cudaStreamDestroy(c.capture);
    if (c.own) cudaStreamDestroy(c.own);
    if (c.pool) cudaMemPoolDestroy(c.pool);
    delete ctx;
    return PHX_OK;
}

int32_t phx_ctx_wait(phx_ctx ctx, uint32_t timeout_ms) {
    if (!ctx) return fail(PHX_ERR_INVALID, "null context");
    PHX_TRY(use(&ctx->c));
    PHX_TRY(wait_stream(ctx->c.stream, timeout_ms));
    return read_status(&ctx->c);
}

void* phx_ctx_stream(phx_ctx ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

int32_t phx_ctx_set_stream(phx_ctx ctx, void* stream) {
    if (!ctx) return fail(PHX_ERR_INVALID, "null context");
    cudaStream_t next = stream ? (cudaStream_t)stream : ctx->c.own;
    if (next != ctx->c.stream) {
        // Frees of the context's memory are ordered on its stream: drain the
        // old one so nothing still running there reads a block freed on the new.
        PHX_TRY(use(&ctx->c));
        PHX_TRY(wait_stream(ctx->c.stream, 0));
    }
    ctx->c.stream = next;
    return PHX_OK;
}

int32_t phx_buf_alloc(phx_ctx ctx, uint64_t bytes, phx_buf* out) {
    if (!ctx || !out) return fail(PHX_ERR_INVALID, "null argument");
    PHX_TRY(use(&ctx->c));
    void* p = nullptr;
    if (bytes) {
        PHX_TRY(ctx_alloc(&ctx->c, &p, bytes));
        int32_t rc = cuda_check(cudaMemsetAsync(p, 0, bytes, ctx->c.stream), "zero");
        if (rc != PHX_OK) {
            ctx_free(&ctx->c, p);
            return rc;
        }
    }
    auto* b = new phx_buf_s();
    b->ctx = &ctx->c;
    b->ptr = p;
    b->bytes = bytes;
    b->owned = true;
    ctx->c.live++;
    *out = b;
    return PHX_OK;
}

int32_t phx_buf_wrap(phx_ctx ctx, void* device_ptr, uint64_t bytes, phx_buf* out) {
    if (!ctx || !out || (!device_ptr && bytes)) return fail(PHX_ERR_INVALID, "null argument");
    auto* b = new phx_buf_s();
    b->ctx = &ctx->c;
    b->ptr = device_ptr;
    b->bytes = bytes;
    b->owned = false;
    ctx->c.live++;
    *out = b;
    return PHX_OK;
}

int32_t phx_buf_free(phx_buf buf) {
    if (!buf) return PHX_OK;
    if (buf->owned && buf->ptr) {
        use(buf->ctx);
        cudaStreamSynchronize(buf->ctx->stream);
        ctx_free(buf->ctx, buf->ptr);
    }
    buf->ctx->live--;
    delete buf;
    return PHX_OK;
}

int32_t phx_buf_write(phx_buf buf, uint64_t offset, const void* src, uint64_t bytes) {
    if (!buf || (!src && bytes)) return fail(PHX_ERR_INVALID, "null argument");
    if (offset + bytes > buf->bytes) return fail(PHX_ERR_INVALID, "write %llu+%llu past %llu bytes",
                                                 (unsigned long long)offset, (unsigned long long)bytes,
                                                 (unsigned long long)buf->bytes);
    if (!bytes) return PHX_OK;
    PHX_TRY(use(buf->ctx));
    PHX_CUDA(cudaMemcpyAsync((char*)buf->ptr + offset, src, bytes, cudaMemcpyHostToDevice, buf->ctx->stream));
    // The source is the caller's and may be reused on return: wait for the
    // copy (a pageable copy is staged anyway; a pinned one is not).
    return wait_stream(buf->ctx->stream, 0);
}

int32_t phx_buf_assign(phx_buf buf, const void* src, uint64_t bytes, int32_t* reallocated) {
    if (!buf || (!src && bytes)) return fail(PHX_ERR_INVALID, "null argument");
    int32_t re = 0;
    if (bytes > buf->bytes) {
        if (!buf->owned) return fail(PHX_ERR_INVALID, "cannot grow a wrapped buffer");
        PHX_TRY(use(buf->ctx));
        cudaStreamSynchronize(buf->ctx->stream);
        void* p = nullptr;
        PHX_TRY(ctx_alloc(buf->ctx, &p, bytes));
        ctx_free(buf->ctx, buf->ptr);
        buf->ptr = p;
        buf->bytes = bytes;
        re = 1;
    }
    if (reallocated) *reallocated = re;
    return phx_buf_write(buf, 0, src, bytes);
}

int32_t phx_buf_read(phx_buf buf, uint64_t offset, void* dst, uint64_t bytes, uint32_t timeout_ms) {
    if (!buf || (!dst && bytes)) return fail(PHX_ERR_INVALID, "null argument");
    if (offset + bytes > buf->bytes) return fail(PHX_ERR_INVALID, "read past the buffer");
    if (!bytes) return PHX_OK;
    PHX_TRY(use(buf->ctx));
    PHX_CUDA(cudaMemcpyAsync(dst, (const char*)buf->ptr + offset, bytes, cudaMemcpyDeviceToHost, buf->ctx->stream));
    return wait_stream(buf->ctx->stream, timeout_ms);
}

uint64_t phx_buf_size(phx_buf buf) { return buf ? buf->bytes : 0; }
void* phx_buf_ptr(phx_buf buf) { return buf ? buf->ptr : nullptr; }

}  // extern "C"

// ---- Pass: recorded launches replayed as one CUDA graph ----

namespace {

struct KernelInfo {
    int32_t id;
    uint32_t nbufs;
    uint32_t params_len;
};

const KernelInfo KERNELS[] = {
    {PHX_KERNEL_SKIN, 5, sizeof(phx_skin_param)},
    {PHX_KERNEL_DENOISE, 1, sizeof(phx_denoise_param)},
    {PHX_KERNEL_MORTON, 2, sizeof(phx_morton_param)},
    {PHX_KERNEL_KARRAS, 2, sizeof(phx_karras_param)},
    {PHX_KERNEL_REFIT, 4, sizeof(phx_refit_param)},
};

const KernelInfo* kernel_info(int32_t id) {
    for (const auto& k : KERNELS)
        if (k.id == id) return &k;
    return nullptr;
}

// Dispatch::new (src/kernel/mod.rs:108-133): 256-wide blocks, x filled up
// to 65,535 then spilled into y. Only groups_x is reported back (params[1]),
// as phiray's kernels read it; the CUDA launches here use a 1-D grid.
uint32_t groups_x(uint32_t items) {
    uint32_t blocks = items == 0 ? 1 : (items + 255) / 256;
    return blocks < 65535 ? blocks : 65535;
}

struct Step {
    int32_t id;
    uint32_t items;
    std::vector<uint8_t> params;
    std::vector<void*> bufs;
    std::vector<uint64_t> sizes;
};

}  // namespace

struct phx_pass_s {
    Ctx* ctx = nullptr;
    std::vector<Step> steps;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
};

static int32_t launch_step(Ctx* c, cudaStream_t s, const Step& st) {
    void* const* b = st.bufs.data();
    switch (st.id) {
        case PHX_KERNEL_SKIN: return launch_skin_step(s, st.params.data(), b, st.sizes.data(), st.items, c->status);
        case PHX_KERNEL_DENOISE: return launch_denoise_step(s, st.params.data(), b, st.items);
        case PHX_KERNEL_MORTON: return launch_morton_step(s, st.params.data(), b, st.items);
        case PHX_KERNEL_KARRAS: return launch_karras_step(s, st.params.data(), b, st.items);
        case PHX_KERNEL_REFIT: return launch_refit_step(s, st.params.data(), b, st.items);
    }
    return fail(PHX_ERR_INVALID, "unknown kernel id %d", st.id);
}

extern "C" {

int32_t phx_pass_create(phx_ctx ctx, phx_pass* out) {
    if (!ctx || !out) return fail(PHX_ERR_INVALID, "null argument");
    auto* p = new phx_pass_s();
    p->ctx = &ctx->c;
    ctx->c.live++;
    *out = p;
    return PHX_OK;
}

int32_t phx_pass_destroy(phx_pass pass) {
    if (!pass) return PHX_OK;
    if (pass->exec) cudaGraphExecDestroy(pass->exec);
    pass->ctx->live--;
    delete pass;
    return PHX_OK;
}

int32_t phx_pass_add(phx_pass pass, int32_t kernel_id, uint32_t n, uint32_t items, const void* params,
                     uint32_t params_len, const phx_buf* bufs, uint32_t nbufs, uint32_t* step) {
    if (!pass) return fail(PHX_ERR_INVALID, "null pass");
    const KernelInfo* k = kernel_info(kernel_id);
    if (!k) return fail(PHX_ERR_INVALID, "unknown kernel id %d", kernel_id);
    // Pass::add_over asserts the binding count (pass.rs:78).
    if (nbufs != k->nbufs) return fail(PHX_ERR_INVALID, "kernel %d: binding count %u, expected %u", kernel_id, nbufs, k->nbufs);
    if (params_len != k->params_len || !params)
        return fail(PHX_ERR_INVALID, "kernel %d: params are %u bytes, expected %u", kernel_id, params_len, k->params_len);
    Step st;
    st.id = kernel_id;
    st.items = items;
    st.params.assign((const uint8_t*)params, (const uint8_t*)params + params_len);
    uint32_t head[2] = {n, groups_x(items)};
    std::memcpy(st.params.data(), head, sizeof head);
    for (uint32_t i = 0; i < nbufs; i++) {
        if (!bufs || !bufs[i]) return fail(PHX_ERR_INVALID, "null buffer %u", i);
        st.bufs.push_back(bufs[i]->ptr);
        st.sizes.push_back(bufs[i]->bytes);
    }
    pass->steps.push_back(std::move(st));
    pass->dirty = true;
    if (step) *step = (uint32_t)pass->steps.size() - 1;
    return PHX_OK;
}

int32_t phx_pass_set(phx_pass pass, uint32_t step, uint32_t offset, const void* data, uint32_t len) {
    if (!pass || step >= pass->steps.size() || (!data && len)) return fail(PHX_ERR_INVALID, "bad step");
    Step& st = pass->steps[step];
    if ((uint64_t)offset + len > st.params.size()) return fail(PHX_ERR_INVALID, "set past the params");
    std::memcpy(st.params.data() + offset, data, len);
    pass->dirty = true;
    return PHX_OK;
}

int32_t phx_pass_run(phx_pass pass) {
    if (!pass) return fail(PHX_ERR_INVALID, "null pass");
    Ctx* c = pass->ctx;
    PHX_TRY(use(c));
    if (pass->steps.empty()) return PHX_OK;
    if (pass->dirty) {
        // Capture the steps as a graph on the private capture stream, then
        // update the executable graph in place (or instantiate it afresh).
        PHX_CUDA(cudaStreamBeginCapture(c->capture, cudaStreamCaptureModeThreadLocal));
        int32_t rc = PHX_OK;
        for (const Step& st : pass->steps) {
            rc = launch_step(c, c->capture, st);
            if (rc != PHX_OK) break;
        }
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->capture, &g);
        if (rc != PHX_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PHX_CUDA(e);
        bool updated = false;
        if (pass->exec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(pass->exec, g, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(pass->exec);
                pass->exec = nullptr;
            }
        }
        if (!updated) {
            e = cudaGraphInstantiate(&pass->exec, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                return cuda_check(e, "cudaGraphInstantiate");
            }
        }
        cudaGraphDestroy(g);
        pass->dirty = false;
    }
    PHX_CUDA(cudaGraphLaunch(pass->exec, c->stream));
    return PHX_OK;
}

int32_t phx_pass_run_step(phx_pass pass, uint32_t step) {
    if (!pass || step >= pass->steps.size()) return fail(PHX_ERR_INVALID, "bad step");
    PHX_TRY(use(pass->ctx));
    return launch_step(pass->ctx, pass->ctx->stream, pass->steps[step]);
}

int32_t phx_pass_clear(phx_pass pass) {
    if (!pass) return fail(PHX_ERR_INVALID, "null pass");
    pass->steps.clear();
    pass->dirty = true;
    return PHX_OK;
}

uint32_t phx_pass_len(phx_pass pass) { return pass ? (uint32_t)pass->steps.size() : 0; }

uint32_t phx_pass_compiled(phx_pass pass) {
    if (!pass) return 0;
    uint32_t seen = 0, count = 0;
    for (const Step& st : pass->steps) {
        uint32_t bit = 1u << st.id;
        if (!(seen & bit)) {
            seen |= bit;
            count++;
        }
    }
    return count;
}

}  // extern "C"
