// 60-bin instantiation of the wavefront renderer: the reference's fixed spectral bins
// (color/principalspectrum.h:7-9). Built with -fmad=false so that its float arithmetic
// rounds like the reference's own build.
#include "fl_render.cuh"

namespace fl {
template fl_status render_waves<60>(Scene *, const CamDev &, const fl_render_params &, double *, WaveCounters *, RenderProfile *,
                                    cudaStream_t, void *, size_t, const LiRays *);
}
