// phx_sort_codes_static: the stable radix sort of Morton codes with no
// allocation at call time.
//
// Who needs it: code that must not call cudaMalloc — a host that reserved
// its device memory up front and hands the renderer a fixed budget, or a
// frame loop that must not stall (cudaMalloc and cudaFree can wait for the
// whole device). Such callers pass their input and output arrays;
// the sort's working memory (the ping-pong key/value arrays, the digit
// histograms, the tile tickets and the look-back words) comes from one
// array of fixed size compiled into this library.
//
// The cost of that choice: the array below (a little under 10 MB) is held
// on every GPU that loads the library until the process exits, and the
// sort handles at most PHX_SORT_STATIC_MAX keys.
#include <mutex>

#include "lbvh.cuh"

namespace {

constexpr uint32_t MAX_KEYS = PHX_SORT_STATIC_MAX;
constexpr uint32_t TILE = phx::LBVH_TILE;
constexpr uint32_t MAX_TILES = (MAX_KEYS + TILE - 1) / TILE;
constexpr size_t HIST_WORDS = 4 * 256;
constexpr size_t TICKET_WORDS = 16;
constexpr size_t LOOKBACK_WORDS = (size_t)4 * MAX_TILES * 256;
constexpr size_t ZERO_WORDS = HIST_WORDS + TICKET_WORDS + LOOKBACK_WORDS;  // cleared every call
constexpr size_t TOTAL_WORDS = ZERO_WORDS + 2 * (size_t)MAX_KEYS;

// The sort's working memory. In host code this name is only a host-side
// stand-in for the device array: the kernels get the device address that
// cudaGetSymbolAddress returns for it (device_scratch below).
static __device__ __align__(256) uint32_t g_sort_scratch[TOTAL_WORDS];

std::mutex g_lock;
// Device address of g_sort_scratch, per device, looked up once for the life
// of the process. A device reset unloads the module and leaves these stale,
// so the library must not outlive a cudaDeviceReset of a device it sorted on.
uint32_t* g_addr[64] = {};

// The device address of the array on the current device, looked up once per
// device (by the first call on a device; the lookup is a host-side query,
// not a stream operation).
int32_t device_scratch(int device, uint32_t** out) {
    if (device < 0 || device >= 64) return phx::fail(PHX_ERR_INVALID, "device %d out of range", device);
    std::lock_guard<std::mutex> g(g_lock);
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return phx::cuda_check(e, "cudaGetSymbolAddress(sort scratch)");
        g_addr[device] = (uint32_t*)p;
    }
    *out = g_addr[device];
    return PHX_OK;
}

}  // namespace

extern "C" int32_t phx_sort_codes_static(phx_ctx ctx, const uint32_t* codes, uint32_t n, uint32_t* order,
                                         uint32_t* sorted) {
    if (!ctx || (n && (!codes || !order || !sorted))) return phx::fail(PHX_ERR_INVALID, "null argument");
    if (n > MAX_KEYS)
        return phx::fail(PHX_ERR_INVALID, "phx_sort_codes_static sorts at most %u keys (got %u); use phx_sort_codes",
                         MAX_KEYS, n);
    if (n == 0) return PHX_OK;
    phx::Ctx* c = &ctx->c;
    PHX_TRY(phx::use(c));
    uint32_t* base = nullptr;
    PHX_TRY(device_scratch(c->device, &base));
    uint32_t* hist = base;
    uint32_t* tickets = base + HIST_WORDS;
    uint32_t* lookback = tickets + TICKET_WORDS;
    uint32_t* alt_keys = base + ZERO_WORDS;
    uint32_t* alt_vals = alt_keys + MAX_KEYS;
    // The array keeps the last call's contents: the counters start at zero.
    PHX_CUDA(cudaMemsetAsync(base, 0, ZERO_WORDS * 4, c->stream));
    // Launch errors come back here; a look-back wait that gives up inside the
    // kernels sets the context's status word, which the next status read
    // (phx_ctx_wait) reports.
    return phx::enqueue_sort_raw(c, codes, n, order, sorted, alt_keys, alt_vals, hist, tickets, lookback, MAX_TILES);
}
