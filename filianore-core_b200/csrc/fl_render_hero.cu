// Hero-wavelength (4 samples) instantiation of the wavefront renderer; FMA allowed.
#include "fl_render.cuh"

namespace fl {
template fl_status render_waves<4>(Scene *, const CamDev &, const fl_render_params &, double *, WaveCounters *, RenderProfile *,
                                   cudaStream_t, void *, size_t, const LiRays *);
}
