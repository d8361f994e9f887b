/*
 * filianore_gpu.h — C ABI of the B200 (sm_100a) spectral path-tracing backend.
 *
 * The reference (filianore-core, C++17) renders with a per-ray virtual call chain:
 *   application loop -> Integrator::Li            src/filianore/integrators/integrator.h:17-18
 *                    -> Scene::intersect          src/filianore/core/scene.h:24
 *                    -> BVH::intersect            src/filianore/bvh/bvh.h:41 (embree4 rtcIntersect1)
 * A GPU cannot be driven one ray at a time, so this ABI replaces that chain at two
 * granularities:
 *   - batch intersection (fl_trace_closest / fl_trace_occluded) replaces BVH::intersect
 *     and rtcIntersect1 one-for-one, on arrays of rays;
 *   - whole-image rendering (fl_render) replaces the absent application's loop over
 *     pixels and samples that calls PathIntegrator::Li.
 *
 * Conventions (all functions):
 *   - every call returns fl_status: FL_OK (0) or a negative error code; no exceptions
 *     cross the boundary; fl_status_string() names a code, fl_last_error() gives detail;
 *   - handles are opaque; the caller owns every buffer it passes, the library owns the
 *     device memory behind a handle;
 *   - pointers marked "host or device" are interpreted according to the `memory`
 *     argument (FL_MEM_HOST: pageable or pinned host memory, copied inside the call;
 *     FL_MEM_DEVICE: device pointers on the context's device, used in place);
 *   - calls on one handle are serialised by an internal mutex; `stream` may be NULL
 *     (the context's own stream) or a cudaStream_t cast to void*.
 */
#ifndef FILIANORE_GPU_H
#define FILIANORE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FL_API __attribute__((visibility("default")))
#else
#define FL_API
#endif

typedef int32_t fl_status;

enum {
    FL_OK = 0,
    FL_ERR_INVALID = -1,     /* bad argument (null pointer, size, enum value) */
    FL_ERR_OOM = -2,         /* device or host allocation failed */
    FL_ERR_CUDA = -3,        /* a CUDA runtime call failed; fl_last_error has the text */
    FL_ERR_TIMEOUT = -4,     /* a bounded wait (host poll) ran out */
    FL_ERR_TRAVERSAL = -5,   /* a traversal hit its stack or iteration bound; results partial */
    FL_ERR_NOT_READY = -6,   /* serving: job not finished yet */
    FL_ERR_CAPACITY = -7,    /* serving: queue or memory budget full, job not admitted */
    FL_ERR_NO_DEVICE = -8    /* no CUDA device / kernel image missing for this GPU */
};

enum { FL_MEM_HOST = 0, FL_MEM_DEVICE = 1 };

typedef struct fl_context fl_context;
typedef struct fl_scene fl_scene;

/* ------------------------------------------------------------------------- */
/* Spectral tables                                                           */
/* ------------------------------------------------------------------------- */
/*
 * The spectral data are supplied by the caller, exactly as the reference holds them in
 * src/filianore/color/cie.h:8-951 (CIE 1931 2-degree observer at 1 nm over 360..830 nm,
 * and the seven reflectance and seven illuminant RGB-to-spectrum basis curves sampled at
 * 32 wavelengths over 380..720 nm). A reference-side integration passes those arrays
 * directly (CIE_Wavelength, CIE_X, ..., RGBRefl2SpectWhite, ...). The library derives
 * the 60-bin tables the reference builds in InitializeSpectrals
 * (src/filianore/color/spectruminits.cpp:6-64) from them.
 * Basis order in refl[] / illum[]: white, cyan, magenta, yellow, red, green, blue.
 */
typedef struct {
    const float *cie_lambda; /* n_cie wavelengths (nm) */
    const float *cie_x;
    const float *cie_y;
    const float *cie_z;
    int32_t n_cie;           /* 471 in the reference */
    float cie_y_integral;    /* 106.856895 in the reference (cie.h:11) */
    const float *rgb2spec_lambda; /* n_rgb2spec wavelengths (nm) */
    int32_t n_rgb2spec;      /* 32 in the reference */
    const float *refl[7];
    const float *illum[7];
    /* Measured metal eta / k curves as the reference holds them in color/metallurgy.h
     * (Gold_Lambda, Gold_Eta, Gold_K, Gold_nSamples, ...), in GetMetalCoefficientsFromForge's
     * order: gold, copper, silver, aluminium, beryllium, chromium, mercury, iridium, lithium.
     * The library bins them as InitializeForge does (color/metallurgy.cpp:7-39). n_metals = 0
     * leaves every metal at eta = k = 0, which is what the reference renders: nothing in it
     * calls InitializeForge, so its metal spectra stay zero (a conductor Fresnel of 1). */
    int32_t n_metals;        /* 0 or 9 */
    int32_t metal_n[9];
    const float *metal_lambda[9];
    const float *metal_eta[9];
    const float *metal_k[9];
} fl_spectral_tables;

/* ------------------------------------------------------------------------- */
/* Context                                                                   */
/* ------------------------------------------------------------------------- */
/* Replaces the global InitializeSpectrals() call (spectruminits.cpp:6) plus embree's
 * rtcNewDevice (bvh.h:25-28): binds a CUDA device, uploads the spectral tables. */
FL_API fl_status fl_context_create(int32_t device, const fl_spectral_tables *tables, fl_context **out);
/* Destroy every scene, guide and server made from the context first: while any is alive
 * the call returns FL_ERR_INVALID and the context stays valid. */
FL_API fl_status fl_context_destroy(fl_context *ctx);
FL_API const char *fl_status_string(fl_status status);
/* Copies the last error message of this context (or of the process when ctx is NULL). */
FL_API fl_status fl_last_error(const fl_context *ctx, char *buf, size_t buf_len);

/* The 60-bin tables the library derived from the caller's tables, for inspection:
 * out has room for 17*60 floats in the order X, Y, Z, refl[0..6], illum[0..6]; with room for
 * 17*60 + 9*120 floats the binned metals follow (per metal: eta, then k). */
FL_API fl_status fl_context_binned_tables(const fl_context *ctx, float *out, size_t n_floats);

/* ------------------------------------------------------------------------- */
/* Scene                                                                     */
/* ------------------------------------------------------------------------- */
enum {
    FL_MAT_LAMBERT = 0,          /* LambertMaterial            shading/materials/lambert.cpp:9-17 */
    FL_MAT_CONDUCTOR = 1,        /* GGX MicrofacetReflection + FresnelConductor
                                    shading/bxdfs/microfacetreflection.cpp, fresnel/fresnelconductor.cpp */
    FL_MAT_ROUGH_DIELECTRIC = 2, /* GGX reflection + MicrofacetTransmission, FresnelDielectric
                                    shading/closures/microfacettransmission.cpp */
    FL_MAT_SMOOTH_DIELECTRIC = 3, /* FresnelSpecular             shading/closures/fresnelspecular.cpp */
    FL_MAT_STANDARD = 4          /* StandardSurfaceMaterial      shading/materials/standardsurface.cpp:72-159;
                                    parameters in fl_scene_desc.standard_surfaces[fl_material.standard] */
};

enum {
    FL_FRESNEL_DIELECTRIC = 0,      /* FresnelType::Dielectric: Schlick with r0 from the specular IOR */
    FL_FRESNEL_METALLIC = 1,        /* FresnelType::Metallic: Schlick with r0 = the specular colour */
    FL_FRESNEL_MEASURED_METAL = 2   /* FresnelType::WavelengthDependentMetallic: FresnelConductor with
                                       the measured eta / k of metal_type (fl_spectral_tables) */
};

/* The StandardSurfaceMaterial's parameters with constant textures. Colours are upsampled
 * with from_reflectance_rgb. The lobes follow compute_scattering_functions, in its order:
 *   - Oren-Nayar diffuse (sigma = 90 kd_roughness) when kd_weight > 0 and either ks_weight
 *     <= 0 or the measured-metal Fresnel; thin_walled turns it into diffuse transmission
 *     (DiffuseTransmission: the same Oren-Nayar lobe, sampled on the far side);
 *   - with ks_weight > 0: FresnelSpecular with R = ks, T = kt when kt_weight > 0; else GGX
 *     (alphas from ks_roughness and ks_anisotropic) with the measured-metal conductor
 *     Fresnel, or the Fresnel-blended diffuse + specular lobe (Schlick dielectric/metallic);
 *   - with thin_film_thickness > 0: GGX with the thin-film interference Fresnel
 *     (ThinFilmInteference(thin_film_ior, thickness in nm, ks_ior));
 *   - an Estevez sheen lobe and a GTR1 clear coat when their weights are > 0.
 * Not supported: bump maps. */
typedef struct {
    float kd[3], kd_weight, kd_roughness;
    float ks[3], ks_weight, ks_roughness, ks_anisotropic, ks_ior;
    int32_t fresnel_type;        /* FL_FRESNEL_* (other values are rejected) */
    int32_t metal_type;          /* FL_FRESNEL_MEASURED_METAL: 0 gold, 1 copper, 2 silver, 3 aluminium,
                                    4 beryllium, 5 chromium, 6 mercury, 7 iridium, 8 lithium; other
                                    values gold, as GetMetalCoefficientsFromForge does */
    float kt[3], kt_weight;
    float sheen_color[3], sheen_weight, sheen_roughness;
    float coat_color[3], coat_weight, coat_ior, coat_gloss;
    float thin_film_thickness, thin_film_ior;
    int32_t thin_walled;
    int32_t kd_texture;          /* 1 + index into fl_scene_desc.images: kd is that ImageMapTexture; 0: kd */
    int32_t bump_texture;        /* 1 + index into fl_scene_desc.images: the bump map, its height the red
                                    byte / 255 of the texel (ImageMapTexture's rule); 0: none. The
                                    shading normal follows Material::bump_evaluate (materials/
                                    material.cpp:8-31) over dpdu, dpdv from the vertex uvs as
                                    Triangle::intersect computes them (shapes/triangle.cpp:33-52) */
} fl_standard_surface;

typedef struct {
    int32_t type;       /* FL_MAT_* */
    float rgb[3];       /* reflectance (Lambert albedo / conductor tint / dielectric tint), upsampled
                           with from_reflectance_rgb (color/spectrumoperations.cpp:113-147) */
    float roughness;    /* alpha = roughness^2 (materials/standardsurface.cpp:104-106) */
    float eta;          /* dielectric IOR, or conductor eta */
    float k;            /* conductor absorption */
    int32_t standard;   /* FL_MAT_STANDARD: index into fl_scene_desc.standard_surfaces */
    int32_t texture;    /* FL_MAT_LAMBERT: 1 + index into fl_scene_desc.images, the reflectance is that
                           ImageMapTexture; 0: rgb */
} fl_material;

/* An RGB image for ImageMapTexture (shading/textures/imagemap.cpp:24-62): width x height
 * pixels of 3 bytes, rows from the top, as stbi_load returns them. Looked up at the hit's
 * uv by the reference's nearest-texel rule: i = int(u * width), j = int((1 - v) * height -
 * 0.001), each clamped to the image (where the reference, for j past the last row, sets i
 * to height - 1 and reads outside the image, the library clamps j as well), then
 * from_reflectance_rgb of the texel / 255. */
typedef struct {
    int32_t width, height;
    const uint8_t *rgb;
} fl_image;

enum {
    FL_LIGHT_TRIANGLE = 0, /* DiffuseAreaIlluminant over one scene triangle (illuminants/diffusearea.cpp) */
    FL_LIGHT_SPHERE = 1,   /* analytic sphere emitter (no reference class) */
    FL_LIGHT_ENV = 2,      /* constant environment radiance (no reference class) */
    FL_LIGHT_POINT = 3,    /* PointIlluminant (illuminants/point.cpp) */
    FL_LIGHT_SPOT = 4,     /* SpotIlluminant (illuminants/spot.cpp) */
    FL_LIGHT_DIRECTIONAL = 5 /* DirectionalIlluminant (illuminants/directional.cpp) */
};

/* Point and spot lights fall off as the squared distance whatever their decay setting: the
 * reference's Illuminant::evaluate_decay_rate (illuminant.cpp:16-35) falls through its switch
 * to d^2. Delta lights take no part in MIS (integrator.cpp:57-61, 66). */
typedef struct {
    int32_t type;          /* FL_LIGHT_* */
    uint32_t tri;          /* FL_LIGHT_TRIANGLE: index of the emitting triangle in the soup */
    float radiance;        /* constant spectral radiance (color * intensity in the reference) */
    float radius;          /* FL_LIGHT_SPHERE */
    float center[3];       /* FL_LIGHT_SPHERE: centre; FL_LIGHT_POINT / SPOT: position */
    float direction[3];    /* FL_LIGHT_SPOT: axis the light shines along; FL_LIGHT_DIRECTIONAL: direction
                              the light travels (the reference's dirIllum constructor argument) */
    float cone_angle;      /* FL_LIGHT_SPOT: outer angle from the axis, radians (after the reference's
                              degree and half-angle options) */
    float penumbra_angle;  /* FL_LIGHT_SPOT: angle from the axis inside which the intensity is full */
} fl_light;

typedef struct {
    const float *verts;             /* n_tri * 9 floats: v0.xyz v1.xyz v2.xyz, FP32 soup */
    uint32_t n_tri;
    const uint32_t *tri_material;   /* n_tri material indices, NULL = all 0 */
    const fl_material *materials;
    uint32_t n_materials;
    const fl_light *lights;         /* order = the reference's Scene::illuminants order */
    uint32_t n_lights;
    const fl_standard_surface *standard_surfaces;  /* for FL_MAT_STANDARD materials (nullable) */
    uint32_t n_standard_surfaces;
    /* Texture coordinates: 6 floats per triangle, (u, v) of its three vertices (nullable).
     * A hit at barycentrics (b1, b2) has uv = uv0 (1 - b1 - b2) + uv1 b1 + uv2 b2. The
     * reference's BVH::intersect leaves uv at (0, 0); without uvs every hit has that uv. */
    const float *uvs;
    const fl_image *images;         /* textures (nullable) */
    uint32_t n_images;
} fl_scene_desc;

typedef struct {
    uint32_t n_tri;
    uint32_t n_nodes;          /* wide (8-ary) BVH nodes */
    uint32_t n_leaves;
    uint32_t max_depth;        /* deepest wide level */
    uint64_t bvh_bytes;        /* node + triangle arrays in HBM */
    double build_ms;           /* device build time (CUDA events) */
} fl_scene_info;

/* Replaces Scene::Scene + BVH::initialize_scene_geometry/finalise (core/scene.cpp:7-19,
 * bvh/bvh.cpp:7-47): uploads the soup (host pointers) and builds the 8-wide BVH on the
 * device. Triangle ids reported by traces are soup indices (= embree geomID order). */
FL_API fl_status fl_scene_create(fl_context *ctx, const fl_scene_desc *desc, fl_scene **out);
FL_API fl_status fl_scene_destroy(fl_scene *scene);
FL_API fl_status fl_scene_get_info(const fl_scene *scene, fl_scene_info *info);

/* ------------------------------------------------------------------------- */
/* Batch ray queries                                                         */
/* ------------------------------------------------------------------------- */
/* Rays are SoA of float4: org_tmin[4*i..] = (ox, oy, oz, tmin), dir_tmax[4*i..] = (dx, dy, dz, tmax).
 * A hit is 16 bytes: int32 triangle id (-1 = miss), float t, float u, float v where
 * p = (1-u-v)*v0 + u*v1 + v*v2 (embree's barycentric convention). Intersection is
 * watertight and double-sided; a hit needs tmin < t < tmax; equal t resolves to the
 * lower triangle id. */
typedef struct {
    int32_t id;
    float t, u, v;
} fl_hit;

/* Replaces BVH::intersect / rtcIntersect1 (bvh/bvh.cpp:49-84) for n rays. */
FL_API fl_status fl_trace_closest(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n,
                           fl_hit *hits, int32_t memory, void *stream);

/* Shadow query with the reference's visibility rule (illuminants/illuminant.cpp:40-50):
 * occluded[i] = 0 when the ray hits nothing in (tmin, tmax) or its closest hit is an
 * emissive triangle, else 1. */
FL_API fl_status fl_trace_occluded(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n,
                            uint8_t *occluded, int32_t memory, void *stream);

/* Traversal statistics of the last trace on this scene (device counters, instrumented
 * launch): total wide nodes and triangles visited. */
FL_API fl_status fl_trace_count(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n,
                         int32_t memory, uint64_t *nodes_visited, uint64_t *tris_tested);

/* ------------------------------------------------------------------------- */
/* Rendering                                                                 */
/* ------------------------------------------------------------------------- */
/* PhysicalCamera (cameras/physical.h:11-43) with aperture 0 (a pinhole) and
 * flipCameraDirection = true, the orientation in which it looks towards look_at (with
 * false it faces away from look_at). Image column 0 lies towards -u, u = up x forward. */
typedef struct {
    float position[3];
    float look_at[3];
    float up[3];
    float vfov_deg;
    int32_t width, height;
    /* PhysicalCamera's aperture: the lens diameter (lensRadius = aperture / 2), focused at
     * the look-at distance; 0 is a pinhole. With a lens, each sample draws two more numbers
     * after (ux, uy, u_lambda) and maps them to the lens with concentric_sample_disk
     * (core/shadingcore.h:65-80). The reference's random_point_on_lens
     * (cameras/physical.cpp:4-10) rejects points outside the disk without drawing new ones,
     * so it never returns for 21% of lens samples. */
    float aperture;
} fl_camera;

enum {
    FL_SPECTRAL_HERO4 = 0,  /* 4 hero wavelengths in 380..720 nm, rotation by 85 nm */
    FL_SPECTRAL_BINS60 = 1  /* the reference's 60 fixed bins over 400..700 nm (principalspectrum.h:7-9) */
};

enum {
    FL_RENDER_PROFILE = 1,  /* time each kernel class with CUDA events (fl_render_stats.ms_*) */
    FL_RENDER_COUNT = 2,    /* count BVH nodes and triangles visited (instrumented traversal) */
    FL_RENDER_CORRECTED_GGX = 4, /* corrected GGX: the density of the visible normals the sampler draws,
                                   sampled on wo's side (the reference keeps D |cos| and the upper
                                   hemisphere, microfacet.cpp:14-16, ggx.cpp:32-57) */
    FL_RENDER_LOBE_DEPTHS = 8    /* depths per sampled lobe kind (diffuse_depth, reflection_depth,
                                   transmission_depth) instead of max_depth for all three */
};

/* The most bounces a path can take (bounce indices 0..FL_MAX_BOUNCES-1). With unequal lobe
 * depths a path is ended only by the depth of the lobe kind it samples, at that exact
 * bounce, so it can outlive the deepest of them until Russian roulette ends it; a path
 * still going at this bound is cut, counted in fl_render_stats.paths_cut, and the call
 * returns FL_ERR_TRAVERSAL (the image holds everything else). */
#define FL_MAX_BOUNCES 250

typedef struct {
    int32_t spp;            /* samples per pixel */
    int32_t max_depth;      /* RenderParams diffuse = reflection = transmission depth (core/renderparams.h:5-10),
                               0..249; ignored with FL_RENDER_LOBE_DEPTHS */
    float rr_threshold;     /* PathIntegrator rrThreshold (pathintegrator.h:11-12), 1 by default */
    int32_t spectral_mode;  /* FL_SPECTRAL_* */
    int32_t wave_paths;     /* path slots of the streaming wave (0 = library default: 2^23 with hero
                               wavelengths, 2^21 with 60 bins); a frame's paths stream through them */
    uint32_t sample_offset; /* first sample index (progressive / multi-GPU sample split) */
    int32_t flags;          /* FL_RENDER_* */
    int32_t reserved;
    /* FL_RENDER_LOBE_DEPTHS: RenderParams' three depths (core/renderparams.h:5-10), each 0..249.
     * PathIntegrator::Li (integrators/pathintegrator.cpp:55-65) ends a path at bounce b when
     * the lobe it sampled there is diffuse and b == diffuse_depth, specular or glossy and
     * b == reflection_depth, or a transmission and b == transmission_depth. */
    int32_t diffuse_depth;
    int32_t reflection_depth;
    int32_t transmission_depth;
    int32_t reserved2;
} fl_render_params;

typedef struct {
    uint64_t paths;          /* camera samples completed */
    uint64_t rays;           /* all rays traced: camera + continuation + shadow + MIS */
    uint64_t shadow_rays;    /* shadow + MIS rays */
    uint64_t bounces;        /* path vertices shaded */
    double ms;               /* device time of the render (CUDA events) */
    uint32_t traversal_errors;
    uint32_t launches;       /* kernels launched by this call */
    /* FL_RENDER_PROFILE: summed device time per kernel class */
    double ms_trace;         /* camera / continuation rays */
    double ms_shade;
    double ms_shadow;        /* shadow + MIS rays */
    double ms_continue;
    /* FL_RENDER_COUNT: traversal work of all rays */
    uint64_t nodes_visited;
    uint64_t tris_tested;
    uint64_t paths_cut;      /* paths ended at FL_MAX_BOUNCES (only with unequal lobe depths) */
} fl_render_stats;

/* Renders the image: for pixel p and sample s the PCG32 stream is seeded with
 * (initstate = p, initseq = 1) and advanced by s * 2^16 draws. film_rgb receives
 * width*height*3 linear Rec.709 floats (the mean over samples of
 * xyz_to_rgb(to_xyz(Li)), color/spectrumoperations.cpp:58-66,193-212), row 0 at the top.
 * film_xyz64 (nullable) receives the FP64 XYZ sums (not divided by spp). */
FL_API fl_status fl_render(fl_scene *scene, const fl_camera *camera, const fl_render_params *params,
                    float *film_rgb, double *film_xyz64, int32_t memory, fl_render_stats *stats);

/* Integrator::Li (integrators/integrator.h:17-18; PathIntegrator::Li,
 * integrators/pathintegrator.cpp:12-87) for a batch of n rays: the radiance each ray brings
 * back. Path i draws its random numbers from its own PCG32 generator (src/ext/pcg32.h) whose
 * 64-bit state the caller passes in rng_state[i], on the reference sampler's default stream
 * (initseq 1, increment 3), in the reference's order (per light: uLight, uScatter; then the
 * BSDF sample; then Russian roulette): the Sampler argument of Li. params: spectral_mode, the
 * depths, rr_threshold and FL_RENDER_CORRECTED_GGX as for fl_render (spp, wave_paths,
 * sample_offset and the other flags are not used). Rays as for fl_trace_closest (the ray's
 * tMin is the third constructor argument of the reference's Ray). lambda0: each ray's hero
 * wavelength in [380, 720) (FL_SPECTRAL_HERO4; ignored, nullable, with 60 bins). Outputs:
 *   radiance  n * 60 floats (FL_SPECTRAL_BINS60, the PrincipalSpectrum Li returns) or n * 4
 *             (the hero wavelengths' samples)
 *   rng_out   the generator state after the path (nullable): the sampler after Li returns
 *   xyz       to_xyz of each radiance (nullable), n * 3 doubles, what fl_render's film adds
 * All pointers are host or device memory according to `memory`. The per-ray form of the
 * reference is this call with n = 1 (slow: one launch sequence per call). */
FL_API fl_status fl_li(fl_scene *scene, const fl_render_params *params, const float *org_tmin, const float *dir_tmax,
                       const uint64_t *rng_state, const float *lambda0, uint32_t n, float *radiance,
                       uint64_t *rng_out, double *xyz, int32_t memory);

/* ------------------------------------------------------------------------- */
/* Serving: continuous batching of render jobs (no counterpart in the reference) */
/* ------------------------------------------------------------------------- */
/* A server keeps registered scenes resident in HBM under a memory budget (least recently
 * used idle scenes are evicted and rebuilt on demand), admits jobs in arrival order as
 * films and scenes fit, and renders the running jobs' samples together: one streaming wave
 * runs continuously, the scheduler appends each plan of samples (about a wave of
 * wave_paths, split over the running jobs by the policy) to it, and a job completes when
 * all its paths have finished. A job's image is the one fl_render gives for the same
 * scene, camera and parameters (hero mode). */
typedef struct fl_server fl_server;

typedef struct {
    uint64_t memory_budget_bytes; /* resident scenes + films of running jobs */
    int32_t wave_paths;           /* path slots of the streaming wave shared by running jobs (0 = 2^21) */
    int32_t max_depth;            /* deepest job accepted */
    int32_t max_jobs;             /* jobs running at once, 1..64 */
    int32_t max_lights;           /* most lights any scene may have, 0..64 */
    int32_t policy;               /* FL_SERVE_*: how each plan of samples is split over the jobs */
} fl_server_config;

enum {
    FL_SERVE_SHORTEST_FIRST = 0,  /* fewest remaining samples first (default) */
    FL_SERVE_FIRST_COME = 1,      /* arrival order */
    FL_SERVE_FAIR_SHARE = 2,      /* equal shares (water-filling) */
    FL_SERVE_SHORTEST_FIRST_AGED = 3, /* shortest first, oldest job keeps a quarter of each wave */
    FL_SERVE_RESPONSE_RATIO = 4,  /* highest (waves waited + waves needed) / waves needed first */
    FL_SERVE_DEADLINE = 5,        /* earliest deadline first, deadline = submission + 2 x the waves the job
                                     needs alone + 1 wave: small jobs pass large ones, a large job's
                                     deadline does not move while it waits */
    FL_SERVE_FIRST_COME_LANE = 6  /* arrival order, with an eighth of each wave reserved for jobs that fit
                                     in it (shortest first): large jobs keep 7/8 of the GPU in arrival
                                     order, small ones do not queue behind them */
};

typedef struct {
    uint64_t scene_id;
    fl_camera camera;
    fl_render_params params;      /* spectral_mode must be FL_SPECTRAL_HERO4 */
} fl_job_desc;

typedef struct {
    double submit_ms, start_ms, done_ms;  /* server clock: submission, admission, image ready */
    uint64_t samples;
} fl_job_stats;

typedef struct {
    uint64_t jobs_submitted, jobs_done, waves, paths, builds, evictions, resident_bytes;
    /* waves: plans of samples appended to the streaming wave; paths: samples planned */
    uint32_t running, pending;
    double busy_ms;               /* host wall time of the graph replays (launch to completion) */
    double wave_max_ms;           /* the longest replay */
    double build_ms, build_max_ms; /* scene builds on the builder thread: total and longest */
    double finish_ms;             /* queueing finished films' resolve and read-out (worker thread) */
    double idle_ms;               /* worker time spent waiting for submissions or builds */
} fl_server_stats;

FL_API fl_status fl_server_create(fl_context *ctx, const fl_server_config *cfg, fl_server **out);
FL_API fl_status fl_server_destroy(fl_server *srv);
/* copies the scene description; the scene is built on the device when a job needs it */
FL_API fl_status fl_server_add_scene(fl_server *srv, const fl_scene_desc *desc, uint64_t *scene_id);
/* The scene takes no more jobs; once no submitted job uses it, its host copy and device
 * arrays are released (for requests that each bring their own scene). */
FL_API fl_status fl_server_remove_scene(fl_server *srv, uint64_t scene_id);
FL_API fl_status fl_server_submit(fl_server *srv, const fl_job_desc *job, uint64_t *job_id);
/* FL_OK and the films (host buffers, nullable) once the job is done, FL_ERR_NOT_READY before;
 * FL_ERR_CAPACITY for a job that can never fit the budget. Results are handed out once. */
FL_API fl_status fl_server_poll(fl_server *srv, uint64_t job_id, float *film_rgb, double *film_xyz64,
                                fl_job_stats *stats);
/* as fl_server_poll, blocking up to timeout_ms (< 0: no limit); FL_ERR_TIMEOUT when it runs out */
FL_API fl_status fl_server_wait(fl_server *srv, uint64_t job_id, int32_t timeout_ms, float *film_rgb,
                                double *film_xyz64, fl_job_stats *stats);
FL_API fl_status fl_server_get_stats(fl_server *srv, fl_server_stats *stats);

/* fl_render_noalloc: fl_render for callers that cannot allocate device memory while they
 * render (an application that owns and budgets all device memory, or code that must not
 * trigger the implicit device synchronisation of cudaMalloc). It has no counterpart in the
 * reference. It allocates nothing: no cudaMalloc/cudaFree, no events, no allocating library
 * call. The path state lives in a fixed 32 MiB device array inside the library (held by
 * every GPU that loads the library until exit); frames stream through as many path slots as
 * fit it, and a scene whose per-path state cannot fit even 128 slots is rejected with
 * FL_ERR_CAPACITY. film_rgb (width*height*3 floats) and film_xyz64 (width*height*3 doubles,
 * the FP64 XYZ sums, cleared by the call) are caller-owned DEVICE buffers. All calls share
 * the fixed array: calls whose GPU work overlaps race and give wrong images. The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress); under CUDA's lazy
 * module loading that is when the driver loads the library code holding the array, which
 * reserves its 32 MiB on the device and may synchronise it. So make the first call during
 * set-up, before any stream capture; later calls allocate nothing. stats->ms is host wall
 * time of the call. */
FL_API fl_status fl_render_noalloc(fl_scene *scene, const fl_camera *camera, const fl_render_params *params,
                                   float *film_rgb, double *film_xyz64, fl_render_stats *stats);

/* ------------------------------------------------------------------------- */
/* Learned path guiding (new: the reference samples directions from the BSDF only) */
/* ------------------------------------------------------------------------- */
/* A guide is an MLP (FP16 weights, FP32 accumulation on the tensor cores) mapping a surface
 * point (12-band frequency encoding of the position in the scene bounds, normal, hero
 * wavelength) through 4 hidden layers of width 64 (ReLU) to an 8-lobe von Mises-Fisher
 * mixture over incident directions. At Lambert vertices the renderer samples the
 * continuation from the mixture with probability select_prob and from the BSDF otherwise,
 * weighting by the one-sample MIS density c q(w) + (1 - c) p_bsdf(w), so images stay
 * unbiased for any weights. Training is online: the renderer records (point, direction,
 * density, incident radiance estimate) at each path's first two Lambert vertices, and
 * after every wave Adam minimises the radiance-weighted KL divergence
 * -E[(L_i cos / p) log q] over minibatches of those records. Hero-wavelength mode only. */
typedef struct fl_guide fl_guide;

typedef struct {
    uint64_t seed;           /* weight initialisation */
    float learning_rate;     /* Adam step size (1e-3 measured steadiest: 1e-2 left some guides worse than none) */
    float select_prob;       /* c in [0, 1): probability of sampling the mixture at a Lambert vertex */
    int32_t batch;           /* records per Adam step, a multiple of 128 in [128, 65536] */
    int32_t max_records;     /* records kept per wave, >= batch */
    int32_t steps_per_wave;  /* most Adam steps after one wave, >= 1 */
    float position_scale;    /* positions enter the encoding as scale * (p - bmin) / (bmax - bmin), in (0, 1];
                                0 means 1. Smaller values shift the 12 bands to coarser frequencies */
    float weight_average;    /* beta in [0, 1): rendering samples from the exponential moving average
                                (decay beta per Adam step, bias-corrected) of the weights Adam
                                produces; 0 renders with Adam's current weights */
    int32_t learn_select;    /* 1: the network also outputs each point's selection probability c, in
                                [0.2, 0.7], fitted with the mixture by minimising -log of the
                                one-sample MIS density c q + (1 - c) p_bsdf; select_prob > 0 still
                                switches guided sampling on. 0: c = select_prob everywhere */
    int32_t train_kernel;    /* FL_GUIDE_TRAIN_*: the kernel of a training step (same gradients) */
} fl_guide_config;

enum {
    FL_GUIDE_TRAIN_MMA_SYNC = 0,  /* warp-level mma.sync (the default: faster at 128 records per CTA) */
    FL_GUIDE_TRAIN_TCGEN05 = 1    /* tcgen05.mma into TMEM for the 128-row products */
};

enum {
    FL_GUIDE_SAMPLE = 1,  /* sample continuations from the guide (one-sample MIS) */
    FL_GUIDE_TRAIN = 2    /* record training samples and take Adam steps after every wave */
};

#define FL_GUIDE_PARAMS 20032   /* weights: [64][80], 3 x [64][64], [41][64], row-major [out][in] */
#define FL_GUIDE_RECORD_FLOATS 20

FL_API fl_status fl_guide_create(fl_context *ctx, const fl_guide_config *cfg, fl_guide **out);
FL_API fl_status fl_guide_destroy(fl_guide *guide);
/* fl_render with guiding (flags FL_GUIDE_*); params->spectral_mode must be FL_SPECTRAL_HERO4. */
FL_API fl_status fl_guide_render(fl_guide *guide, fl_scene *scene, const fl_camera *camera,
                                 const fl_render_params *params, int32_t flags, float *film_rgb,
                                 double *film_xyz64, int32_t memory, fl_render_stats *stats);
/* Renders passes of params->spp samples per pixel until budget_ms of wall time have passed,
 * training during the first train_fraction of the budget and sampling from the guide once it
 * has taken an Adam step. The film is the average of all passes; stats->paths / (width *
 * height) is the number of samples per pixel rendered, stats->ms the wall time. */
FL_API fl_status fl_guide_render_timed(fl_guide *guide, fl_scene *scene, const fl_camera *camera,
                                       const fl_render_params *params, double budget_ms, double train_fraction,
                                       float *film_rgb, double *film_xyz64, int32_t memory,
                                       fl_render_stats *stats);
/* FP32 master weights (FL_GUIDE_PARAMS floats, host). Setting them resets Adam's moments. */
FL_API fl_status fl_guide_get_weights(fl_guide *guide, float *weights);
FL_API fl_status fl_guide_set_weights(fl_guide *guide, const float *weights);
FL_API fl_status fl_guide_get_info(fl_guide *guide, int64_t *adam_steps, float *last_loss);
/* Training loss and its gradient on n host records (FL_GUIDE_RECORD_FLOATS floats each:
 * position 3, normal 3, wavelength, direction 3, density, incident radiance, then 8 unused)
 * in the bounds [bmin, bmax]: grad (FL_GUIDE_PARAMS floats) = d/dweights of
 * mean_i w_i * -log q(direction_i) with w_i = L_i cos_i / density_i / mean(w) (with learn_select,
 * -log(c q + (1 - c) cos_i / pi) in place of -log q). Weights are
 * unchanged. n <= max_records. */
FL_API fl_status fl_guide_gradient(fl_guide *guide, const float *records, uint32_t n, const float bmin[3],
                                   const float bmax[3], float *grad, float *loss);
/* The training records of the last trained wave (at most max_n; *n receives the count),
 * FL_GUIDE_RECORD_FLOATS floats each: position 3, normal 3, wavelength, direction 3,
 * density, incident radiance estimate, path throughput after the vertex [4], radiance
 * gathered before it [4]. */
FL_API fl_status fl_guide_get_records(fl_guide *guide, float *records, uint32_t max_n, uint32_t *n);
/* Mixture parameters (41 floats per record: pi[8], mu[8][3], kappa[8], the learned selection
 * probability c) for the points of n host records in the bounds [bmin, bmax]. */
FL_API fl_status fl_guide_eval(fl_guide *guide, const float *records, uint32_t n, const float bmin[3],
                               const float bmax[3], float *mixture);

#ifdef __cplusplus
}
#endif

#endif /* FILIANORE_GPU_H */
