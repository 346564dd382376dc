// Single-instance render kernels, ids 13-15: the megakernel with the
// per-sample warp wait at 10, 12 and 16 resident blocks.
#include "render.cuh"

namespace phx {

int32_t render_flat_c(uint32_t kernel, bool stats, const RenderLaunch& L) {
    switch (kernel) {
        case PHX_KERNEL_MEGAKERNEL_10_SYNC: return stats ? launch_mk<MODE_STATS, 10, true>(L) : launch_mk<0, 10, true>(L);
        case PHX_KERNEL_MEGAKERNEL_12_SYNC: return stats ? launch_mk<MODE_STATS, 12, true>(L) : launch_mk<0, 12, true>(L);
        default: return stats ? launch_mk<MODE_STATS, 16, true>(L) : launch_mk<0, 16, true>(L);
    }
}

}  // namespace phx
