// Internal host-side state behind the opaque handles of include/filianore_gpu.h.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/filianore_gpu.h"
#include "fl_device.cuh"

namespace fl {

// Device-resident spectral tables (raw tables for hero wavelengths, 60-bin tables for
// the reference's fixed bins). Staged into shared memory by the shading kernels.
struct SpectralTablesDev {
    float cie_lambda0;      // first CIE wavelength (1 nm spacing)
    int n_cie;
    float cie_y_integral;
    float rgb_lambda0, rgb_lambda1;
    int n_rgb;
    float *cie_xyz;         // 3 * n_cie (x, y, z rows)
    float *rgb_bases;       // 14 * n_rgb (refl 0..6, illum 0..6)
    float *binned;          // 17 * 60 (X, Y, Z, refl 0..6, illum 0..6)
};

struct Context {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string last_error;
    std::vector<float> binned_host;  // 17 * 60
    std::vector<float> metal60;      // 9 metals x (eta, k) x 60 bins (zero without metal curves)
    SpectralTablesDev tables{};
    // grow-only scratch owned by the context (render wavefront state, trace staging)
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    void *film_scratch = nullptr;       // render films (separate from the wave scratch)
    size_t film_bytes = 0;
    std::vector<cudaEvent_t> events;    // reusable timing events (FL_RENDER_PROFILE)
    // one wave's launch sequence captured as a CUDA graph, with what it was captured for
    cudaGraphExec_t wave_graph = nullptr;
    const void *graph_base = nullptr;
    size_t graph_cap = 0;
    int graph_depth = -1, graph_nl_mode = -1, graph_count = -1, graph_std = -1;
    std::atomic<int> children{0};       // live scenes, guides and servers made from this context
    int *d_error = nullptr;             // traversal error counter
    unsigned long long *d_counters = nullptr;  // 8 x u64 statistics
    // Stream-ordered pool for scene arrays and BVH build temporaries: allocations and frees
    // are ordered on `stream` without device synchronisation, and freed blocks stay cached
    // for the next scene (up to kPoolKeepBytes).
    cudaMemPool_t pool = nullptr;
    // a second stream for host-memory trace batches (copies of one chunk overlap the
    // traversal of another), and the events that fork it from and join it to the caller's
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};
constexpr uint64_t kPoolKeepBytes = (uint64_t)8 << 30;

// Device material record (constant over the render).
struct MaterialDev {
    int type;
    float rgb[3];
    float ax, ay;
    float eta, k;
    int basis[3];       // Smits basis indices of from_reflectance_rgb
    float w[3];         // and their weights
    int standard;       // FL_MAT_STANDARD: index into Scene::standard
    int texture;        // FL_MAT_LAMBERT: image of its reflectance, -1: rgb
};

// An ImageMapTexture's pixels in Scene::pixels: RGB bytes, rows from the top.
struct ImageDev {
    unsigned long long offset;  // first byte
    int width, height;
};

// StandardSurfaceMaterial with constant textures, reduced on the host to what
// compute_scattering_functions (materials/standardsurface.cpp:72-159) hands its BxDFs.
// Lobe ids: 4 Oren-Nayar, 5 Fresnel-blended diffuse + specular, 6 Estevez sheen,
// 7 GTR1 clear coat, 8 FresnelSpecular with R = ks and T = kt, 9 GGX with the measured-metal
// conductor Fresnel, 10 GGX with the thin-film Fresnel, 11 diffuse transmission.
// Its spectra (kStdSpectra rows of 60 bins in Scene::std_refl60): kd, ks, kt, sheen colour,
// coat colour, metal eta, metal k.
constexpr int kStdSpectra = 7;
struct StandardDev {
    int n_lobes;
    int lobes[5];         // in the order the material adds them
    float eta;            // BSDF::eta: ks_ior with both specular and transmission weights, else 1
    float ior;            // ks_ior (FresnelSpecular, Schlick r0)
    float ax, ay;         // GGX alphas with the anisotropic aspect
    float kd_weight, on_A, on_B;  // OrenNayarBRDF(kd, kdweight, 90 kdrough)
    float fb_A, fb_B;             // the blended lobe's OrenNayarBRDF(kd, kdweight, kdrough)
    float ks_weight, ro;
    int fresnel_type;     // FL_FRESNEL_*
    float sheen_weight, sheen_rough;
    float coat_weight, coat_ior, coat_gloss;  // coat_gloss = lerp(gloss, .1, .001)
    float tf_ior, tf_thickness;                // thin film over a medium of IOR ior
    int kd_texture;                            // image of kd, -1: the constant kd
    int bump_texture;                          // bump map image (red channel), -1: none
    int basis[5][3];      // Smits terms of kd, ks, kt, sheen colour, coat colour
    float w[5][3];
};

struct LightDev {
    int type;
    uint32_t tri;
    float radiance;
    float radius;
    float cx, cy, cz;   // sphere centre, point / spot position
    float area;         // triangle or sphere area
    float dx, dy, dz;   // spot axis (as given); directional: normalize(-travel direction), towards the light
    float cos_cone, cos_penumbra;  // spot
};

struct Scene {
    Context *ctx = nullptr;
    bool counted = false;  // included in ctx->children
    uint32_t n_tri = 0;
    uint32_t n_nodes = 0;
    uint32_t n_leaves = 0;
    uint32_t max_depth = 0;
    double build_ms = 0.0;
    WideNode *nodes = nullptr;        // n_nodes
    float4 *tris = nullptr;           // 3 * n_tri, BVH order
    float *soup = nullptr;            // 9 * n_tri, soup order (hit records, light sampling)
    uint32_t *tri_material = nullptr; // soup order
    int32_t *tri_light = nullptr;     // soup order, -1 = not emissive
    MaterialDev *materials = nullptr;
    float *mat_refl60 = nullptr;      // n_materials x 60: from_reflectance_rgb in the 60 bins
    StandardDev *standard = nullptr;  // n_standard StandardSurface records
    float *std_refl60 = nullptr;      // n_standard x kStdSpectra x 60: their spectra in the 60 bins
    uint32_t n_standard = 0;
    float *uvs = nullptr;             // 6 per triangle, soup order (null: every hit has uv (0, 0))
    unsigned char *pixels = nullptr;  // the images' RGB bytes
    ImageDev *images = nullptr;
    uint32_t n_images = 0;
    bool ext_kernels = false;         // StandardSurface or image-textured materials: their kernel instances run
    uint32_t n_materials = 0;
    LightDev *lights = nullptr;
    uint32_t n_lights = 0;
    uint32_t n_emissive_tris = 0;
    int has_env = 0;
    float env_radiance = 0.f;
    float bmin[3] = {0.f, 0.f, 0.f}, bmax[3] = {0.f, 0.f, 0.f};  // bounds of the triangles
    std::vector<fl_light> lights_host;
    std::vector<MaterialDev> materials_host;
};

// error plumbing -----------------------------------------------------------------------
void set_error(Context *ctx, const std::string &msg);
fl_status cuda_status(Context *ctx, cudaError_t e, const char *what);

#define FL_CUDA_TRY(ctx, call)                                    \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return cuda_status(ctx, _e, #call); \
    } while (0)

// BVH build (fl_bvh_build.cu): builds nodes/tris of `s` from s->soup on ctx->stream.
fl_status build_bvh(Scene *s);

// traversal launches (fl_trace.cu); arrays are device pointers.
enum TraceKind { kTraceClosest = 0, kTraceOccluded = 1, kTraceCount = 2 };
// fetch_slot (0 or 1) picks the launch's work counter: launches that may run at the same
// time on different streams use different slots.
fl_status launch_trace(Scene *s, const float4 *org_tmin, const float4 *dir_tmax, uint32_t n, fl_hit *hits,
                       uint8_t *occluded, int kind, cudaStream_t stream, int fetch_slot);

// device memory from the context's pool, ordered on ctx->stream
fl_status dev_alloc(Context *ctx, void **p, size_t bytes);
void dev_free(Context *ctx, void *p);
template <typename T>
fl_status dev_alloc_n(Context *ctx, T **p, size_t count) {
    return dev_alloc(ctx, reinterpret_cast<void **>(p), sizeof(T) * (count ? count : 1));
}

// context scratch: returns a device buffer of at least `bytes` (grow-only)
fl_status ensure_scratch(Context *ctx, size_t bytes, void **out);
fl_status ensure_film_scratch(Context *ctx, size_t bytes, void **out);

// RenderParams' three depths (core/renderparams.h:5-10) in the order diffuse, reflection
// (specular and glossy), transmission: the params' own with FL_RENDER_LOBE_DEPTHS, else
// max_depth for all three.
inline void lobe_depths(const fl_render_params &p, int d[3]) {
    if (p.flags & FL_RENDER_LOBE_DEPTHS) {
        d[0] = p.diffuse_depth;
        d[1] = p.reflection_depth;
        d[2] = p.transmission_depth;
    } else {
        d[0] = d[1] = d[2] = p.max_depth;
    }
}
// every depth a bounce index below FL_MAX_BOUNCES
inline bool depths_ok(const fl_render_params &p) {
    int d[3];
    lobe_depths(p, d);
    for (int k = 0; k < 3; ++k)
        if (d[k] < 0 || d[k] >= FL_MAX_BOUNCES) return false;
    return true;
}
// Equal depths end every path at that bounce (a sampled lobe is always diffuse, glossy or
// specular); unequal ones let paths run on (fl_render.cuh, run_tail).
inline bool depths_equal(const fl_render_params &p) {
    int d[3];
    lobe_depths(p, d);
    return d[0] == d[1] && d[1] == d[2];
}
// the bounces a wave's fixed launch sequence covers: 0..deepest depth
inline int deepest_depth(const fl_render_params &p) {
    int d[3];
    lobe_depths(p, d);
    return std::max(d[0], std::max(d[1], d[2]));
}

// camera resolution within 2^31 pixels and a finite, non-negative aperture
inline bool camera_ok(const fl_camera &c) {
    return c.width > 0 && c.height > 0 && (uint64_t)c.width * c.height <= (1ull << 31) && c.aperture >= 0.f &&
           c.aperture <= 3.0e38f;
}

// Smits terms of from_reflectance_rgb (color/spectrumoperations.cpp:113-147): basis ids
// (0 white, 1 cyan, 2 magenta, 3 yellow, 4 red, 5 green, 6 blue) and weights, in its order.
__host__ __device__ inline void smits_terms(const float rgb[3], int basis[3], float w[3]) {
    if (rgb[0] <= rgb[1] && rgb[0] <= rgb[2]) {
        basis[0] = 0; w[0] = rgb[0];
        if (rgb[1] <= rgb[2]) { basis[1] = 1; w[1] = rgb[1] - rgb[0]; basis[2] = 6; w[2] = rgb[2] - rgb[1]; }
        else { basis[1] = 1; w[1] = rgb[2] - rgb[0]; basis[2] = 5; w[2] = rgb[1] - rgb[2]; }
    } else if (rgb[1] <= rgb[0] && rgb[1] <= rgb[2]) {
        basis[0] = 0; w[0] = rgb[1];
        if (rgb[0] <= rgb[2]) { basis[1] = 2; w[1] = rgb[0] - rgb[1]; basis[2] = 6; w[2] = rgb[2] - rgb[0]; }
        else { basis[1] = 2; w[1] = rgb[2] - rgb[1]; basis[2] = 4; w[2] = rgb[0] - rgb[2]; }
    } else {
        basis[0] = 0; w[0] = rgb[2];
        if (rgb[0] <= rgb[1]) { basis[1] = 3; w[1] = rgb[0] - rgb[2]; basis[2] = 5; w[2] = rgb[1] - rgb[0]; }
        else { basis[1] = 3; w[1] = rgb[1] - rgb[2]; basis[2] = 4; w[2] = rgb[0] - rgb[1]; }
    }
}

}  // namespace fl
