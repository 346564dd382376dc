// Single-instance render kernels, ids 0 and 4-8: the megakernel at 4, 3, 2
// and 5 resident blocks, with and without the per-sample warp wait.
#include "render.cuh"

namespace phx {

int32_t render_flat_a(uint32_t kernel, bool stats, const RenderLaunch& L) {
    switch (kernel) {
        case PHX_KERNEL_MEGAKERNEL_3: return stats ? launch_mk<MODE_STATS, 3, false>(L) : launch_mk<0, 3, false>(L);
        case PHX_KERNEL_MEGAKERNEL_2: return stats ? launch_mk<MODE_STATS, 2, false>(L) : launch_mk<0, 2, false>(L);
        case PHX_KERNEL_MEGAKERNEL_SYNC: return stats ? launch_mk<MODE_STATS, 4, true>(L) : launch_mk<0, 4, true>(L);
        case PHX_KERNEL_MEGAKERNEL_2_SYNC: return stats ? launch_mk<MODE_STATS, 2, true>(L) : launch_mk<0, 2, true>(L);
        case PHX_KERNEL_MEGAKERNEL_5: return stats ? launch_mk<MODE_STATS, 5, false>(L) : launch_mk<0, 5, false>(L);
        default: return stats ? launch_mk<MODE_STATS, 4, false>(L) : launch_mk<0, 4, false>(L);
    }
}

}  // namespace phx
