// The full-mode render kernels: scenes of instances and frames that draw the
// floor grid, in the three forms launch_placed maps kernel ids to.
#include "render.cuh"

namespace phx {

int32_t render_full(uint32_t kernel, bool stats, const RenderLaunch& L) {
    return stats ? launch_placed<MODE_FULL | MODE_STATS>(kernel, L) : launch_placed<MODE_FULL>(kernel, L);
}

}  // namespace phx
