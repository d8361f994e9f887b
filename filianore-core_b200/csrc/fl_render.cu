// fl_render: whole-image rendering through the wavefront kernels (fl_render.cuh).
#include <algorithm>
#include <cmath>

#include "fl_render.cuh"

namespace fl {
extern template fl_status render_waves<4>(Scene *, const CamDev &, const fl_render_params &, double *, WaveCounters *,
                                          RenderProfile *, cudaStream_t, void *, size_t, const LiRays *);
extern template fl_status render_waves<60>(Scene *, const CamDev &, const fl_render_params &, double *,
                                           WaveCounters *, RenderProfile *, cudaStream_t, void *, size_t,
                                           const LiRays *);

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
    if (!camera_ok(*camera) || p.spp <= 0 || !depths_ok(p) ||
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
        stats->paths_cut = hc.cut;
    }
    return render_bounds_status(ctx, hc);
}

extern "C" fl_status fl_li(fl_scene *scene_h, const fl_render_params *params, const float *org_tmin,
                           const float *dir_tmax, const uint64_t *rng_state, const float *lambda0, uint32_t n,
                           float *radiance, uint64_t *rng_out, double *xyz, int32_t memory) {
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!s) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!params) {
        set_error(ctx, "null parameters");
        return FL_ERR_INVALID;
    }
    const fl_render_params p = *params;
    const bool hero = p.spectral_mode == FL_SPECTRAL_HERO4;
    if (!depths_ok(p) || (!hero && p.spectral_mode != FL_SPECTRAL_BINS60) ||
        (memory != FL_MEM_HOST && memory != FL_MEM_DEVICE) || n >= (1u << 31)) {
        set_error(ctx, "invalid Li parameters");
        return FL_ERR_INVALID;
    }
    if (n == 0) return FL_OK;
    if (!org_tmin || !dir_tmax || !rng_state || !radiance || (hero && !lambda0)) {
        set_error(ctx, "null ray, generator, wavelength or radiance buffer");
        return FL_ERR_INVALID;
    }
    if (s->n_lights > 64) {
        set_error(ctx, "more than 64 lights");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int NL = hero ? 4 : 60;
    // device buffers: the film scratch holds the XYZ sums and, for host pointers, the staged
    // inputs and outputs (the wave state lives in the context scratch)
    const bool host = memory == FL_MEM_HOST;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t b_xyz = al((size_t)n * 3 * sizeof(double));
    const size_t b_ray = al((size_t)n * 16), b_rng = al((size_t)n * 8), b_lam = al((size_t)n * 4);
    const size_t b_L = al((size_t)n * NL * 4);
    const size_t total = b_xyz + (host ? 2 * b_ray + 2 * b_rng + b_lam + b_L : 0);
    void *fs = nullptr;
    fl_status rc = ensure_film_scratch(ctx, total, &fs);
    if (rc) return rc;
    char *B = static_cast<char *>(fs);
    double *d_xyz = (xyz && !host) ? xyz : reinterpret_cast<double *>(B);
    LiRays li{};
    if (host) {
        char *q = B + b_xyz;
        float4 *o = reinterpret_cast<float4 *>(q);
        float4 *d = reinterpret_cast<float4 *>(q + b_ray);
        unsigned long long *r = reinterpret_cast<unsigned long long *>(q + 2 * b_ray);
        unsigned long long *ro = reinterpret_cast<unsigned long long *>(q + 2 * b_ray + b_rng);
        float *lam = reinterpret_cast<float *>(q + 2 * b_ray + 2 * b_rng);
        float *L = reinterpret_cast<float *>(q + 2 * b_ray + 2 * b_rng + b_lam);
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(o, org_tmin, (size_t)n * 16, cudaMemcpyHostToDevice, st));
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(d, dir_tmax, (size_t)n * 16, cudaMemcpyHostToDevice, st));
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(r, rng_state, (size_t)n * 8, cudaMemcpyHostToDevice, st));
        if (hero) FL_CUDA_TRY(ctx, cudaMemcpyAsync(lam, lambda0, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        li = LiRays{o, d, r, hero ? lam : nullptr, L, ro};
    } else {
        li = LiRays{reinterpret_cast<const float4 *>(org_tmin), reinterpret_cast<const float4 *>(dir_tmax),
                    reinterpret_cast<const unsigned long long *>(rng_state), hero ? lambda0 : nullptr, radiance,
                    reinterpret_cast<unsigned long long *>(rng_out)};
    }
    FL_CUDA_TRY(ctx, cudaMemsetAsync(d_xyz, 0, (size_t)n * 3 * sizeof(double), st));
    // ray i is pixel i of a one-sample job: a camera of n x 1 pixels that k_raygen never reads
    CamDev cam{};
    cam.W = (int)n;
    cam.H = 1;
    fl_render_params q = p;
    q.spp = 1;
    q.sample_offset = 0;
    q.wave_paths = 0;
    q.flags = p.flags & (FL_RENDER_CORRECTED_GGX | FL_RENDER_LOBE_DEPTHS);
    WaveCounters hc{};
    RenderProfile prof;
    rc = hero ? render_waves<4>(s, cam, q, d_xyz, &hc, &prof, st, nullptr, 0, &li)
              : render_waves<60>(s, cam, q, d_xyz, &hc, &prof, st, nullptr, 0, &li);
    if (rc) return rc;
    if (host) {
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(radiance, li.L, (size_t)n * NL * 4, cudaMemcpyDeviceToHost, st));
        if (rng_out) FL_CUDA_TRY(ctx, cudaMemcpyAsync(rng_out, li.rng_out, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
        if (xyz) FL_CUDA_TRY(ctx, cudaMemcpyAsync(xyz, d_xyz, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return render_bounds_status(ctx, hc);
}
