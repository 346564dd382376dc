// The wavefront render's kernels in every mode.
#include "render.cuh"

namespace phx {

uint32_t wf_slot_words() { return WF_WORDS; }

int32_t render_wavefront(bool full, bool stats, const RenderLaunch& L, const WfBuffers& B) {
    if (full) return stats ? launch_wf<MODE_FULL | MODE_STATS>(L, B) : launch_wf<MODE_FULL>(L, B);
    return stats ? launch_wf<MODE_STATS>(L, B) : launch_wf<0>(L, B);
}

}  // namespace phx
