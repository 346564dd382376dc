// Single-instance render kernels, ids 9-12: the megakernel at 6 and 8
// resident blocks, with and without the per-sample warp wait.
#include "render.cuh"

namespace phx {

int32_t render_flat_b(uint32_t kernel, bool stats, const RenderLaunch& L) {
    switch (kernel) {
        case PHX_KERNEL_MEGAKERNEL_6_SYNC: return stats ? launch_mk<MODE_STATS, 6, true>(L) : launch_mk<0, 6, true>(L);
        case PHX_KERNEL_MEGAKERNEL_8: return stats ? launch_mk<MODE_STATS, 8, false>(L) : launch_mk<0, 8, false>(L);
        case PHX_KERNEL_MEGAKERNEL_8_SYNC: return stats ? launch_mk<MODE_STATS, 8, true>(L) : launch_mk<0, 8, true>(L);
        default: return stats ? launch_mk<MODE_STATS, 6, false>(L) : launch_mk<0, 6, false>(L);
    }
}

}  // namespace phx
