// fl_render: whole-image rendering through the wavefront kernels (fl_render.cuh).
#include <algorithm>
#include <cmath>

#include "fl_render.cuh"

namespace fl {
extern template fl_status render_waves<4>(Scene *, const CamDev &, const fl_render_params &, double *, WaveCounters *,
                                          RenderProfile *, cudaStream_t, void *, size_t);
extern template fl_status render_waves<60>(Scene *, const CamDev &, const fl_render_params &, double *,
                                           WaveCounters *, RenderProfile *, cudaStream_t, void *, size_t);

// PhysicalCamera::PhysicalCamera (cameras/physical.h:11-43) with aperture 0 and
// flipCameraDirection = true (the orientation that faces look_at).
CamDev camera_basis_of(const fl_camera &c) {
    const v3 pos = mk(c.position[0], c.position[1], c.position[2]);
    const v3 at = mk(c.look_at[0], c.look_at[1], c.look_at[2]);
    const v3 up = mk(c.up[0], c.up[1], c.up[2]);
    const float focusDistance = len(sub(pos, at));
    const float theta = c.vfov_deg * kPi / 180.f;
    const float halfHeight = tanf(theta / 2.f);
    const float aspect = (float)c.width / (float)c.height;
    const float halfWidth = aspect * halfHeight;
    v3 w = normalize(sub(pos, at));
    w = mul(w, -1.f);
    const v3 u = normalize(cross(up, w));
    const v3 v = cross(w, u);
    w = mul(w, -1.f);
    CamDev d;
    d.origin = pos;
    d.u = u;
    d.v = v;
    d.lower_left = sub(sub(sub(pos, mul(mul(u, halfWidth), focusDistance)), mul(mul(v, focusDistance), halfHeight)),
                       mul(w, focusDistance));
    d.horizontal = mul(mul(mul(u, 2.f), halfWidth), focusDistance);
    d.vertical = mul(mul(mul(v, 2.f), halfHeight), focusDistance);
    d.W = c.width;
    d.H = c.height;
    d.lens_radius = c.aperture / 2.f;
    return d;
}
}  // namespace fl

using namespace fl;

extern "C" fl_status fl_render(fl_scene *scene_h, const fl_camera *camera, const fl_render_params *params,
                               float *film_rgb, double *film_xyz64, int32_t memory, fl_render_stats *stats) {
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!s) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!camera || !params || !film_rgb) {
        set_error(ctx, "null camera, parameters or film");
        return FL_ERR_INVALID;
    }
    const fl_render_params p = *params;
    if (!camera_ok(*camera) || p.spp <= 0 || p.max_depth < 0 || p.max_depth > 250 ||
        (p.spectral_mode != FL_SPECTRAL_HERO4 && p.spectral_mode != FL_SPECTRAL_BINS60) ||
        (memory != FL_MEM_HOST && memory != FL_MEM_DEVICE)) {
        set_error(ctx, "invalid render parameters");
        return FL_ERR_INVALID;
    }
    if (s->n_lights > 64) {
        set_error(ctx, "more than 64 lights");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const CamDev cam = camera_basis_of(*camera);
    const size_t n_pix = (size_t)camera->width * camera->height;
    // film scratch: FP64 XYZ sums (unless the caller's device buffer is used) + FP32 RGB staging
    const bool own_xyz = !(film_xyz64 && memory == FL_MEM_DEVICE);
    const size_t xyz_bytes = (n_pix * 3 * sizeof(double) + 255) & ~(size_t)255;
    void *fs = nullptr;
    fl_status rc = ensure_film_scratch(ctx, xyz_bytes + n_pix * 3 * sizeof(float), &fs);
    if (rc) return rc;
    double *d_xyz = own_xyz ? static_cast<double *>(fs) : film_xyz64;
    float *d_rgb = memory == FL_MEM_DEVICE ? film_rgb : reinterpret_cast<float *>(static_cast<char *>(fs) + xyz_bytes);
    FL_CUDA_TRY(ctx, cudaMemsetAsync(d_xyz, 0, n_pix * 3 * sizeof(double), st));
    cudaEvent_t e0, e1;
    FL_CUDA_TRY(ctx, cudaEventCreate(&e0));
    FL_CUDA_TRY(ctx, cudaEventCreate(&e1));
    FL_CUDA_TRY(ctx, cudaEventRecord(e0, st));
    WaveCounters hc{};
    RenderProfile prof;
    prof.on = (p.flags & FL_RENDER_PROFILE) != 0;
    prof.pool = &ctx->events;
    rc = p.spectral_mode == FL_SPECTRAL_BINS60 ? render_waves<60>(s, cam, p, d_xyz, &hc, &prof, st)
                                               : render_waves<4>(s, cam, p, d_xyz, &hc, &prof, st);
    if (rc) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
    }
    k_resolve<<<std::min<size_t>((n_pix + 255) / 256, (size_t)ctx->sm_count * 8), 256, 0, st>>>(
        d_xyz, (uint32_t)n_pix, 1.0 / (double)p.spp, d_rgb);
    FL_CUDA_TRY(ctx, cudaGetLastError());
    FL_CUDA_TRY(ctx, cudaEventRecord(e1, st));
    if (memory == FL_MEM_HOST) {
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(film_rgb, d_rgb, n_pix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (film_xyz64)
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(film_xyz64, d_xyz, n_pix * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        stats->paths = hc.paths;
        stats->rays = hc.rays;
        stats->shadow_rays = hc.shadow_rays;
        stats->bounces = hc.bounces;
        stats->ms = ms;
        stats->traversal_errors = (uint32_t)hc.err;
        stats->launches = prof.launches + 1;
        double cls[4] = {0, 0, 0, 0};
        if (prof.on) prof.sum(cls);
        stats->ms_trace = cls[0];
        stats->ms_shade = cls[1];
        stats->ms_shadow = cls[2];
        stats->ms_continue = cls[3];
        stats->nodes_visited = hc.nodes;
        stats->tris_tested = hc.tris;
    }
    if (hc.err) {
        set_error(ctx, std::to_string(hc.err) + " traversal or queue bound hits during the render");
        return FL_ERR_TRAVERSAL;
    }
    return FL_OK;
}
