// Single-instance render kernels, ids 1-3: the persistent state machine at
// 4, 6 and 8 resident blocks.
#include "render.cuh"

namespace phx {

int32_t render_flat_sm(uint32_t kernel, bool stats, const RenderLaunch& L) {
    switch (kernel) {
        case PHX_KERNEL_STATE_MACHINE_6: return stats ? launch_sm<MODE_STATS, 6>(L) : launch_sm<0, 6>(L);
        case PHX_KERNEL_STATE_MACHINE_8: return stats ? launch_sm<MODE_STATS, 8>(L) : launch_sm<0, 8>(L);
        default: return stats ? launch_sm<MODE_STATS, 4>(L) : launch_sm<0, 4>(L);
    }
}

}  // namespace phx
