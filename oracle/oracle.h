/*
 * ORACLE — test infrastructure only. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load liboracle.so, and only as the checker or the timed
 * CPU baseline; the product library (filianore-core_b200) never links or calls it.
 *
 * A CPU restatement, in plain C, of the reference's spectral path-tracing hot path:
 * closest-hit ray casting (orc_trace.c), spectral tables and sampling (orc_spectral.c)
 * and the path integrator (orc_render.c). Each function cites the reference lines it
 * restates. Parity is pinned against the reference's own code compiled here
 * (oracle/_ref, built by oracle/Makefile from the sources under the reference tree).
 */
#ifndef ORC_ORACLE_H
#define ORC_ORACLE_H

#include "../include/filianore_gpu.h"
#include "orc_math.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- rays */
typedef struct {
    float o[3], d[3], inv_d[3];
    float tmin, tmax;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    int valid;
} orc_ray;

void orc_ray_precompute(const float *o_tmin, const float *d_tmax, orc_ray *r);
int orc_intersect_watertight(const orc_ray *r, const float *tri9, float *t, float *u, float *v);

typedef struct orc_bvh orc_bvh;
orc_bvh *orc_bvh_build(const float *tris, uint32_t n);
void orc_bvh_free(orc_bvh *b);
uint32_t orc_bvh_node_count(const orc_bvh *b);
int32_t orc_bvh_closest(const orc_bvh *b, const orc_ray *r, float *t, float *u, float *v,
                        uint64_t *nodes_visited, uint64_t *tris_tested);
void orc_trace_closest(const orc_bvh *bvh, const float *org_tmin, const float *dir_tmax, uint32_t n,
                       fl_hit *hits, int nthreads, uint64_t *nodes_visited, uint64_t *tris_tested);
void orc_trace_brute(const float *tris, uint32_t n_tri, const float *org_tmin, const float *dir_tmax,
                     uint32_t n, fl_hit *hits);

/* ---------------------------------------------------------------- PCG32 (src/ext/pcg32.h:40-163) */
typedef struct { uint64_t state, inc; } orc_pcg32;
void orc_pcg32_seed(orc_pcg32 *r, uint64_t initstate, uint64_t initseq);
uint32_t orc_pcg32_next(orc_pcg32 *r);
float orc_pcg32_nextf(orc_pcg32 *r);
void orc_pcg32_advance(orc_pcg32 *r, int64_t delta);
/* n draws of nextUInt after seed(initstate, initseq) and advance(adv), for known-answer tests */
void orc_pcg32_sequence(uint64_t initstate, uint64_t initseq, int64_t adv, uint32_t n, uint32_t *out);

/* ---------------------------------------------------------------- spectra */
#define ORC_NBINS 60
#define ORC_MAXLAMBDA 60
typedef struct {
    /* raw tables (copied from the caller) */
    int n_cie, n_rgb;
    float cie_lambda[512], cie_x[512], cie_y[512], cie_z[512];
    float cie_y_integral;
    float rgb_lambda[64];
    float refl[7][64], illum[7][64];
    /* 60-bin tables built as InitializeSpectrals does (color/spectruminits.cpp:6-64) */
    float X[ORC_NBINS], Y[ORC_NBINS], Z[ORC_NBINS];
    float brefl[7][ORC_NBINS], billum[7][ORC_NBINS];
    /* measured metals binned as InitializeForge does (color/metallurgy.cpp:7-39): eta, k;
     * zero without metal curves (the reference never calls InitializeForge) */
    float metal[9][2][ORC_NBINS];
} orc_tables;

int orc_tables_init(orc_tables *t, const fl_spectral_tables *src);
/* average_spectrum_samples, color/spectrumoperations.cpp:28-56 */
float orc_average_spectrum_samples(const float *lambda, const float *vals, int n, float l0, float l1);
/* 17*60 floats: X, Y, Z, refl[7], illum[7] */
void orc_tables_binned(const orc_tables *t, float *out);
/* the binned metal spectra: 9 metals x (eta, k) x 60 */
void orc_tables_metals(const orc_tables *t, float *out);

/* ---------------------------------------------------------------- render */
typedef struct {
    int nthreads;
    const uint32_t *pixels;  /* optional subset of pixel indices (NULL = all) */
    uint32_t n_pixels;
} orc_render_opts;

typedef struct {
    uint64_t paths, rays, shadow_rays, bounces;
} orc_render_counts;

/* film_xyz: width*height*3 doubles, receives the sums over samples of to_xyz(Li). */
int orc_render(const fl_scene_desc *scene, const orc_tables *tables, const fl_camera *cam,
               const fl_render_params *params, const orc_render_opts *opts, double *film_xyz,
               orc_render_counts *counts);

/* camera basis exactly as PhysicalCamera::PhysicalCamera (cameras/physical.h:11-43) */
typedef struct { v3 origin, lower_left, horizontal, vertical, u, v; float lens_radius; } orc_camera;
void orc_camera_init(const fl_camera *c, orc_camera *out);
/* one camera ray for (pixel, sample) plus the hero-wavelength draw; returns 3 floats used */
void orc_camera_ray(const orc_camera *cam, const fl_camera *c, uint32_t pixel, orc_pcg32 *rng,
                    v3 *o, v3 *d, float *u_lambda);
void orc_camera_rays(const fl_camera *cam, const uint32_t *pixels, uint32_t n, uint32_t sample, float *org_tmin,
                     float *dir_tmax, uint64_t *rng_state, float *lambda0);
int orc_li(const fl_scene_desc *sc, const orc_tables *tab, const fl_render_params *P, uint32_t n,
           const float *org_tmin, const float *dir_tmax, const uint64_t *rng_state, const float *lambda0,
           float *radiance, uint64_t *rng_out, double *xyz);

/* spectral upsampling used by materials: 60 bins or hero wavelengths */
void orc_reflectance(const orc_tables *t, const float rgb[3], int mode, const float *lambda, float *out);
void orc_xyz_from_spectrum(const orc_tables *t, int mode, const float *lambda, const float *L, double *xyz);

/* f(wo, wi) |cos theta_i| of a non-Lambert material in its local frame, n directions */
void orc_bsdf_fcos(const fl_material *m, const float wo[3], uint32_t n, const float *wi, int corrected, float *out);
/* ImageMapTexture's texel rule (RGB / 255) at n uv pairs */
void orc_image_texels(const fl_image *im, const float *uv, uint32_t n, float *rgb);

/* ---------------------------------------------------------------- guiding (orc_guide.c) */
/* 1: evaluate without the GPU's FP16 roundings (for finite-difference checks) */
void orc_guide_set_exact(int on);
/* mixture parameters (40 floats per record) of the guide with FP32 weights w32 */
void orc_guide_eval(const float *w32, const float *rec, uint32_t n, const float bmin[3], const float bmax[3],
                    float *mix);
/* gradient of the weighted training loss (FL_GUIDE_PARAMS floats); returns the mean loss */
float orc_guide_gradient(const float *w32, const float *rec, uint32_t n, const float bmin[3], const float bmax[3],
                         float *grad, int learned);

#ifdef __cplusplus
}
#endif
#endif
