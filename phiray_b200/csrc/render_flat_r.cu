// Single-instance render kernels, ids 17-19: the megakernel whose walk keeps
// the top of its stack in registers: 8 entries at 4 resident blocks (128
// registers a thread), the top entry at 8 and at 16 blocks with the
// per-sample warp wait.
#include "render.cuh"

namespace phx {

int32_t render_flat_r(uint32_t kernel, bool stats, const RenderLaunch& L) {
    constexpr int R8 = MODE_REG | MODE_REG8;
    switch (kernel) {
        case PHX_KERNEL_MEGAKERNEL_8_SYNC_REG:
            return stats ? launch_mk<MODE_STATS | MODE_REG, 8, true>(L) : launch_mk<MODE_REG, 8, true>(L);
        case PHX_KERNEL_MEGAKERNEL_16_SYNC_REG:
            return stats ? launch_mk<MODE_STATS | MODE_REG, 16, true>(L) : launch_mk<MODE_REG, 16, true>(L);
        default: return stats ? launch_mk<MODE_STATS | R8, 4, false>(L) : launch_mk<R8, 4, false>(L);
    }
}

}  // namespace phx
