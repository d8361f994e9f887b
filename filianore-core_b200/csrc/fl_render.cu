// fl_render: whole-image rendering (placeholder until the wavefront kernels land).
#include "fl_render.cuh"

extern "C" fl_status fl_render(fl_scene *scene, const fl_camera *camera, const fl_render_params *params,
                               float *film_rgb, double *film_xyz64, int32_t memory, fl_render_stats *stats) {
    (void)scene; (void)camera; (void)params; (void)film_rgb; (void)film_xyz64; (void)memory; (void)stats;
    return FL_ERR_INVALID;
}
