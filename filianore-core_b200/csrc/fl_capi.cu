// C ABI: contexts, spectral tables, scenes (include/filianore_gpu.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "fl_internal.h"

namespace fl {

namespace {
std::mutex g_err_mu;
std::string g_last_error;  // errors not tied to a context (creation failures)
}  // namespace

void set_error(Context *ctx, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    std::lock_guard<std::mutex> lock(g_err_mu);
    g_last_error = msg;
}

fl_status cuda_status(Context *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return FL_OK;
    set_error(ctx, std::string(what) + ": " + cudaGetErrorString(e));
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return FL_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorNoKernelImageForDevice ||
        e == cudaErrorInsufficientDriver)
        return FL_ERR_NO_DEVICE;
    return FL_ERR_CUDA;
}

// the emissive-triangle table: triangle -> its light (the rest stay -1)
__global__ void k_tri_light(const LightDev *__restrict__ lights, uint32_t n_lights, int32_t *__restrict__ tri_light) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n_lights && lights[l].type == FL_LIGHT_TRIANGLE) tri_light[lights[l].tri] = (int32_t)l;
}

fl_status dev_alloc(Context *ctx, void **p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, ctx->pool, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_status(ctx, e, "device allocation");
    }
    return FL_OK;
}

void dev_free(Context *ctx, void *p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}

fl_status ensure_scratch(Context *ctx, size_t bytes, void **out) {
    if (bytes > ctx->scratch_bytes) {
        if (ctx->wave_graph) {  // captured against the old buffer
            cudaGraphExecDestroy(ctx->wave_graph);
            ctx->wave_graph = nullptr;
            ctx->graph_base = nullptr;
        }
        if (ctx->scratch) {
            cudaStreamSynchronize(ctx->stream);
            if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
            cudaFree(ctx->scratch);
            ctx->scratch = nullptr;
            ctx->scratch_bytes = 0;
        }
        size_t want = bytes + bytes / 4;
        cudaError_t e = cudaMalloc(&ctx->scratch, want);
        if (e != cudaSuccess) return cuda_status(ctx, e, "scratch allocation");
        ctx->scratch_bytes = want;
    }
    *out = ctx->scratch;
    return FL_OK;
}

fl_status ensure_film_scratch(Context *ctx, size_t bytes, void **out) {
    if (bytes > ctx->film_bytes) {
        if (ctx->film_scratch) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->film_scratch);
            ctx->film_scratch = nullptr;
            ctx->film_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&ctx->film_scratch, bytes);
        if (e != cudaSuccess) return cuda_status(ctx, e, "film allocation");
        ctx->film_bytes = bytes;
    }
    *out = ctx->film_scratch;
    return FL_OK;
}

// average_spectrum_samples (src/filianore/color/spectrumoperations.cpp:28-56), with the
// reference's float/double mixing, so the 60-bin tables equal InitializeSpectrals'.
static float lerp_ref(float t, float v1, float v2) { return (1.f - t) * v1 + t * v2; }

float average_spectrum_samples(const float *wl, const float *vals, int n, float ws, float we) {
    if (we <= wl[0]) return vals[0];
    if (ws >= wl[n - 1]) return vals[n - 1];
    if (n == 1) return vals[0];
    float sum = 0;
    if (ws < wl[0]) sum += vals[0] * (wl[0] - ws);
    if (we > wl[n - 1]) sum += vals[n - 1] * (we - wl[n - 1]);
    int i = 0;
    while (ws > wl[i + 1]) ++i;
    for (; i + 1 < n && we >= wl[i]; ++i) {
        const float ss = std::max(ws, wl[i]);
        const float se = std::min(we, wl[i + 1]);
        const float ia = lerp_ref((ss - wl[i]) / (wl[i + 1] - wl[i]), vals[i], vals[i + 1]);
        const float ib = lerp_ref((se - wl[i]) / (wl[i + 1] - wl[i]), vals[i], vals[i + 1]);
        sum = (float)((double)sum + 0.5 * (double)(ia + ib) * (double)(se - ss));
    }
    return sum / (we - ws);
}


// from_reflectance_rgb (color/spectrumoperations.cpp:113-147) over the 60 bins, clamped
// at zero (spectrum_clamp) from the Smits terms
static void refl60(const std::vector<float> &binned, const int basis[3], const float w[3], float *out) {
    for (int i = 0; i < 60; ++i) {
        float r = 0.f;
        for (int k = 0; k < 3; ++k) r += binned[180 + 60 * basis[k] + i] * w[k];
        r *= 0.94f;
        out[i] = r < 0.f ? 0.f : r;
    }
}

// OrenNayarBRDF's A and B from sigma in degrees (bxdfs/orennayar.cpp:6-12)
static void oren_nayar_ab(float sigma_deg, float *A, float *B) {
    const float sigma = (kPi / 180.f) * sigma_deg;
    const float sigma2 = sigma * sigma;
    *A = 1.f - (sigma2 / (2.f * (sigma2 + 0.33f)));
    *B = 0.45f * sigma2 / (sigma2 + 0.09f);
}

// StandardSurfaceMaterial::compute_scattering_functions (materials/standardsurface.cpp:72-159)
// with constant textures: the lobes it adds and their parameters
static StandardDev standard_dev(const fl_standard_surface &P) {
    StandardDev d{};
    d.eta = (P.ks_weight > 0 && P.kt_weight > 0) ? P.ks_ior : 1.f;
    d.ior = P.ks_ior;
    d.kd_weight = P.kd_weight;
    oren_nayar_ab(P.kd_roughness * 90.f, &d.on_A, &d.on_B);  // sigma = 90 kdroughness
    oren_nayar_ab(P.kd_roughness, &d.fb_A, &d.fb_B);         // the blended lobe passes kdroughness as sigma
    const float aspect = std::sqrt(1.f - P.ks_anisotropic * 0.9f);
    const float a2 = P.ks_roughness * P.ks_roughness;
    d.ax = std::max(.001f, a2 / aspect);
    d.ay = std::max(.001f, a2 * aspect);
    d.ro = ((1.f - P.ks_ior) / (1.f + P.ks_ior)) * ((1.f - P.ks_ior) / (1.f + P.ks_ior));
    d.ks_weight = P.ks_weight;
    d.fresnel_type = P.fresnel_type;
    d.sheen_weight = P.sheen_weight;
    d.sheen_rough = std::max(.001f, P.sheen_roughness);
    d.coat_weight = P.coat_weight;
    d.coat_ior = P.coat_ior;
    d.coat_gloss = (1.f - P.coat_gloss) * .1f + P.coat_gloss * .001f;  // lerp(gloss, .1, .001)
    d.tf_ior = P.thin_film_ior;
    d.tf_thickness = P.thin_film_thickness;
    const bool measured = P.fresnel_type == FL_FRESNEL_MEASURED_METAL;
    d.n_lobes = 0;
    if ((P.kd_weight > 0 && P.ks_weight <= 0) || (P.kd_weight > 0 && P.ks_weight > 0 && measured))
        d.lobes[d.n_lobes++] = P.thin_walled ? 11 : 4;  // DiffuseTransmission or OrenNayarBRDF
    if (P.ks_weight > 0) d.lobes[d.n_lobes++] = P.kt_weight > 0 ? 8 : (measured ? 9 : 5);
    if (P.thin_film_thickness > 0) d.lobes[d.n_lobes++] = 10;
    if (P.sheen_weight > 0) d.lobes[d.n_lobes++] = 6;
    if (P.coat_weight > 0) d.lobes[d.n_lobes++] = 7;
    const float *rgb[5] = {P.kd, P.ks, P.kt, P.sheen_color, P.coat_color};
    for (int c = 0; c < 5; ++c) smits_terms(rgb[c], d.basis[c], d.w[c]);
    return d;
}

}  // namespace fl

using namespace fl;

extern "C" {

const char *fl_status_string(fl_status s) {
    switch (s) {
    case FL_OK: return "FL_OK";
    case FL_ERR_INVALID: return "FL_ERR_INVALID";
    case FL_ERR_OOM: return "FL_ERR_OOM";
    case FL_ERR_CUDA: return "FL_ERR_CUDA";
    case FL_ERR_TIMEOUT: return "FL_ERR_TIMEOUT";
    case FL_ERR_TRAVERSAL: return "FL_ERR_TRAVERSAL";
    case FL_ERR_NOT_READY: return "FL_ERR_NOT_READY";
    case FL_ERR_CAPACITY: return "FL_ERR_CAPACITY";
    case FL_ERR_NO_DEVICE: return "FL_ERR_NO_DEVICE";
    default: return "FL_ERR_UNKNOWN";
    }
}

fl_status fl_last_error(const fl_context *ctx_h, char *buf, size_t n) {
    if (!buf || n == 0) return FL_ERR_INVALID;
    const Context *ctx = reinterpret_cast<const Context *>(ctx_h);
    std::string msg;
    if (ctx) msg = ctx->last_error;
    else {
        std::lock_guard<std::mutex> lock(g_err_mu);
        msg = g_last_error;
    }
    std::snprintf(buf, n, "%s", msg.c_str());
    return FL_OK;
}

fl_status fl_context_create(int32_t device, const fl_spectral_tables *t, fl_context **out) {
    if (!out) return FL_ERR_INVALID;
    *out = nullptr;
    if (!t || !t->cie_lambda || !t->cie_x || !t->cie_y || !t->cie_z || t->n_cie < 2 || t->n_cie > 512 ||
        !t->rgb2spec_lambda || t->n_rgb2spec < 2 || t->n_rgb2spec > 64) {
        set_error(nullptr, "incomplete spectral tables");
        return FL_ERR_INVALID;
    }
    for (int b = 0; b < 7; ++b)
        if (!t->refl[b] || !t->illum[b]) {
            set_error(nullptr, "missing RGB-to-spectrum basis");
            return FL_ERR_INVALID;
        }
    if (t->n_metals != 0 && t->n_metals != 9) {
        set_error(nullptr, "n_metals must be 0 or 9");
        return FL_ERR_INVALID;
    }
    for (int m = 0; m < t->n_metals; ++m)
        if (t->metal_n[m] < 1 || t->metal_n[m] > 4096 || !t->metal_lambda[m] || !t->metal_eta[m] || !t->metal_k[m]) {
            set_error(nullptr, "incomplete metal curve");
            return FL_ERR_INVALID;
        }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error(nullptr, "no CUDA device");
        return FL_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) {
        set_error(nullptr, "device index out of range");
        return FL_ERR_INVALID;
    }
    Context *ctx = new Context();
    ctx->device = device;
    fl_status rc;
#define CTX_TRY(call)                                        \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) {                             \
            rc = cuda_status(nullptr, _e, #call);            \
            fl_context_destroy(reinterpret_cast<fl_context *>(ctx)); \
            return rc;                                       \
        }                                                    \
    } while (0)
    CTX_TRY(cudaSetDevice(device));
    CTX_TRY(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
    CTX_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        CTX_TRY(cudaMemPoolCreate(&ctx->pool, &props));
        uint64_t keep = kPoolKeepBytes;
        CTX_TRY(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    CTX_TRY(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CTX_TRY(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
    CTX_TRY(cudaMalloc(&ctx->d_error, sizeof(int) * 4));
    CTX_TRY(cudaMalloc(&ctx->d_counters, sizeof(unsigned long long) * 8));

    // 60-bin tables as InitializeSpectrals builds them (color/spectruminits.cpp:6-64), and
    // the metals as InitializeForge does (color/metallurgy.cpp:7-39)
    ctx->binned_host.assign(17 * 60, 0.f);
    ctx->metal60.assign(9 * 120, 0.f);
    for (int i = 0; i < 60; ++i) {
        const float wl0 = lerp_ref((float)i / 60.f, 400.f, 700.f);
        const float wl1 = lerp_ref((float)(i + 1) / 60.f, 400.f, 700.f);
        ctx->binned_host[i] = average_spectrum_samples(t->cie_lambda, t->cie_x, t->n_cie, wl0, wl1);
        ctx->binned_host[60 + i] = average_spectrum_samples(t->cie_lambda, t->cie_y, t->n_cie, wl0, wl1);
        ctx->binned_host[120 + i] = average_spectrum_samples(t->cie_lambda, t->cie_z, t->n_cie, wl0, wl1);
        for (int b = 0; b < 7; ++b) {
            ctx->binned_host[180 + 60 * b + i] =
                average_spectrum_samples(t->rgb2spec_lambda, t->refl[b], t->n_rgb2spec, wl0, wl1);
            ctx->binned_host[600 + 60 * b + i] =
                average_spectrum_samples(t->rgb2spec_lambda, t->illum[b], t->n_rgb2spec, wl0, wl1);
        }
        for (int m = 0; m < t->n_metals; ++m) {
            ctx->metal60[120 * m + i] = average_spectrum_samples(t->metal_lambda[m], t->metal_eta[m], t->metal_n[m], wl0, wl1);
            ctx->metal60[120 * m + 60 + i] =
                average_spectrum_samples(t->metal_lambda[m], t->metal_k[m], t->metal_n[m], wl0, wl1);
        }
    }
    SpectralTablesDev &T = ctx->tables;
    T.cie_lambda0 = t->cie_lambda[0];
    T.n_cie = t->n_cie;
    T.cie_y_integral = t->cie_y_integral;
    T.rgb_lambda0 = t->rgb2spec_lambda[0];
    T.rgb_lambda1 = t->rgb2spec_lambda[t->n_rgb2spec - 1];
    T.n_rgb = t->n_rgb2spec;
    std::vector<float> cie(3 * (size_t)t->n_cie), bases(14 * (size_t)t->n_rgb2spec);
    std::memcpy(cie.data(), t->cie_x, sizeof(float) * t->n_cie);
    std::memcpy(cie.data() + t->n_cie, t->cie_y, sizeof(float) * t->n_cie);
    std::memcpy(cie.data() + 2 * t->n_cie, t->cie_z, sizeof(float) * t->n_cie);
    for (int b = 0; b < 7; ++b) {
        std::memcpy(bases.data() + (size_t)b * t->n_rgb2spec, t->refl[b], sizeof(float) * t->n_rgb2spec);
        std::memcpy(bases.data() + (size_t)(7 + b) * t->n_rgb2spec, t->illum[b], sizeof(float) * t->n_rgb2spec);
    }
    CTX_TRY(cudaMalloc(&T.cie_xyz, sizeof(float) * cie.size()));
    CTX_TRY(cudaMalloc(&T.rgb_bases, sizeof(float) * bases.size()));
    CTX_TRY(cudaMalloc(&T.binned, sizeof(float) * 17 * 60));
    CTX_TRY(cudaMemcpy(T.cie_xyz, cie.data(), sizeof(float) * cie.size(), cudaMemcpyHostToDevice));
    CTX_TRY(cudaMemcpy(T.rgb_bases, bases.data(), sizeof(float) * bases.size(), cudaMemcpyHostToDevice));
    CTX_TRY(cudaMemcpy(T.binned, ctx->binned_host.data(), sizeof(float) * 17 * 60, cudaMemcpyHostToDevice));
#undef CTX_TRY
    *out = reinterpret_cast<fl_context *>(ctx);
    return FL_OK;
}

fl_status fl_context_destroy(fl_context *ctx_h) {
    Context *ctx = reinterpret_cast<Context *>(ctx_h);
    if (!ctx) return FL_ERR_INVALID;
    if (ctx->children.load() != 0) {
        // scenes, guides or servers still refer to this context: keep it alive rather than
        // leave them dangling
        set_error(ctx, "context still has live scenes, guides or servers");
        return FL_ERR_INVALID;
    }
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
    if (ctx->wave_graph) cudaGraphExecDestroy(ctx->wave_graph);
    cudaFree(ctx->scratch);
    cudaFree(ctx->film_scratch);
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->tables.cie_xyz);
    cudaFree(ctx->tables.rgb_bases);
    cudaFree(ctx->tables.binned);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->stream2) {
        cudaStreamSynchronize(ctx->stream2);
        cudaStreamDestroy(ctx->stream2);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return FL_OK;
}

fl_status fl_context_binned_tables(const fl_context *ctx_h, float *out, size_t n) {
    const Context *ctx = reinterpret_cast<const Context *>(ctx_h);
    if (!ctx || !out || n < 17 * 60) return FL_ERR_INVALID;
    std::memcpy(out, ctx->binned_host.data(), sizeof(float) * 17 * 60);
    if (n >= 17 * 60 + 9 * 120) std::memcpy(out + 17 * 60, ctx->metal60.data(), sizeof(float) * 9 * 120);
    return FL_OK;
}

// Frees a scene (the caller holds ctx->mu). Every entry point returns with its work
// finished, so nothing in flight reads the scene; the arrays go back to the context's pool
// in stream order.
static void scene_release(Scene *s) {
    Context *ctx = s->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    void *arrays[] = {s->nodes, s->tris, s->soup, s->tri_material, s->tri_light, s->materials, s->lights,
                      s->mat_refl60, s->standard, s->std_refl60, s->uvs, s->pixels, s->images};
    for (void *p : arrays) dev_free(ctx, p);
    if (s->counted) s->ctx->children--;
    delete s;
}

fl_status fl_scene_create(fl_context *ctx_h, const fl_scene_desc *d, fl_scene **out) {
    Context *ctx = reinterpret_cast<Context *>(ctx_h);
    if (!ctx || !d || !out) return FL_ERR_INVALID;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if ((d->n_tri && !d->verts) || (d->n_lights && !d->lights) || (d->n_materials == 0 || !d->materials)) {
        set_error(ctx, "scene needs vertices for its triangles and at least one material");
        return FL_ERR_INVALID;
    }
    for (uint32_t i = 0; i < d->n_materials; ++i) {
        const fl_material &M = d->materials[i];
        if (M.type < FL_MAT_LAMBERT || M.type > FL_MAT_STANDARD) {
            set_error(ctx, "unknown material type");
            return FL_ERR_INVALID;
        }
        if (M.type == FL_MAT_STANDARD &&
            (!d->standard_surfaces || M.standard < 0 || (uint32_t)M.standard >= d->n_standard_surfaces)) {
            set_error(ctx, "standard surface index out of range");
            return FL_ERR_INVALID;
        }
        if (M.texture < 0 || (M.texture > 0 && (!d->images || (uint32_t)M.texture > d->n_images))) {
            set_error(ctx, "material texture index out of range");
            return FL_ERR_INVALID;
        }
    }
    for (uint32_t i = 0; d->images && i < d->n_images; ++i) {
        const fl_image &im = d->images[i];
        if (im.width <= 0 || im.height <= 0 || !im.rgb || (uint64_t)im.width * im.height > (1ull << 28)) {
            set_error(ctx, "invalid image (needs pixels, at most 2^28 of them)");
            return FL_ERR_INVALID;
        }
    }
    for (uint32_t i = 0; d->standard_surfaces && i < d->n_standard_surfaces; ++i) {
        const fl_standard_surface &P = d->standard_surfaces[i];
        if (P.fresnel_type != FL_FRESNEL_DIELECTRIC && P.fresnel_type != FL_FRESNEL_METALLIC &&
            P.fresnel_type != FL_FRESNEL_MEASURED_METAL) {
            set_error(ctx, "standard surface: unknown fresnel_type");
            return FL_ERR_INVALID;
        }
        if (P.kd_texture < 0 || (P.kd_texture > 0 && (!d->images || (uint32_t)P.kd_texture > d->n_images)) ||
            P.bump_texture < 0 || (P.bump_texture > 0 && (!d->images || (uint32_t)P.bump_texture > d->n_images))) {
            set_error(ctx, "standard surface: texture index out of range");
            return FL_ERR_INVALID;
        }
    }
    if (d->tri_material)
        for (uint32_t i = 0; i < d->n_tri; ++i)
            if (d->tri_material[i] >= d->n_materials) {
                set_error(ctx, "triangle material index out of range");
                return FL_ERR_INVALID;
            }
    Scene *s = new Scene();
    s->ctx = ctx;
    s->n_tri = d->n_tri;
    for (int a = 0; a < 3; ++a) s->bmin[a] = s->bmax[a] = 0.f;  // the BVH build sets them
    for (uint32_t l = 0; l < d->n_lights; ++l) {
        const fl_light &L = d->lights[l];
        if (L.type == FL_LIGHT_TRIANGLE) {
            if (L.tri >= d->n_tri) {
                delete s;
                set_error(ctx, "light triangle index out of range");
                return FL_ERR_INVALID;
            }
            s->n_emissive_tris++;
        } else if (L.type == FL_LIGHT_ENV) {
            s->has_env = 1;
            s->env_radiance = L.radiance;
        } else if (L.type == FL_LIGHT_SPOT || L.type == FL_LIGHT_DIRECTIONAL) {
            const float dl = L.direction[0] * L.direction[0] + L.direction[1] * L.direction[1] +
                             L.direction[2] * L.direction[2];
            if (!(dl > 0.f) || !std::isfinite(dl) || !std::isfinite(L.cone_angle) || !std::isfinite(L.penumbra_angle)) {
                delete s;
                set_error(ctx, "spot and directional lights need a direction (and finite angles)");
                return FL_ERR_INVALID;
            }
        } else if (L.type != FL_LIGHT_SPHERE && L.type != FL_LIGHT_POINT) {
            delete s;
            set_error(ctx, "unknown light type");
            return FL_ERR_INVALID;
        }
        s->lights_host.push_back(L);
    }
    std::vector<LightDev> lights_dev;
    for (uint32_t l = 0; l < d->n_lights; ++l) {
        const fl_light &L = d->lights[l];
        LightDev ld{};
        ld.type = L.type;
        ld.tri = L.tri;
        ld.radiance = L.radiance;
        ld.radius = L.radius;
        ld.cx = L.center[0]; ld.cy = L.center[1]; ld.cz = L.center[2];
        if (L.type == FL_LIGHT_TRIANGLE) {
            const float *v = d->verts + 9 * (size_t)L.tri;
            v3 a = mk(v[0], v[1], v[2]), b = mk(v[3], v[4], v[5]), c = mk(v[6], v[7], v[8]);
            ld.area = 0.5f * len(cross(sub(b, a), sub(c, a)));  // Triangle::area, triangle.cpp:130-132
        } else if (L.type == FL_LIGHT_SPHERE) {
            ld.area = 4.f * kPi * L.radius * L.radius;
        } else if (L.type == FL_LIGHT_SPOT) {
            // SpotIlluminant (spot.cpp:6-20): the axis as given, cosines of the angles
            ld.dx = L.direction[0]; ld.dy = L.direction[1]; ld.dz = L.direction[2];
            ld.cos_cone = std::cos(L.cone_angle);
            ld.cos_penumbra = std::cos(L.penumbra_angle);
        } else if (L.type == FL_LIGHT_DIRECTIONAL) {
            // DirectionalIlluminant (directional.cpp:6-12): towards the light, normalised
            const v3 w = normalize(neg(mk(L.direction[0], L.direction[1], L.direction[2])));
            ld.dx = w.x; ld.dy = w.y; ld.dz = w.z;
        }
        lights_dev.push_back(ld);
    }
    for (uint32_t m = 0; m < d->n_materials; ++m) {
        const fl_material &M = d->materials[m];
        MaterialDev md{};
        md.type = M.type;
        md.rgb[0] = M.rgb[0]; md.rgb[1] = M.rgb[1]; md.rgb[2] = M.rgb[2];
        const float a = M.roughness * M.roughness;
        md.ax = md.ay = a > 0.001f ? a : 0.001f;  // GGXDistribution clamps alpha (ggx.cpp:7-10)
        md.eta = M.eta;
        md.k = M.k;
        smits_terms(M.rgb, md.basis, md.w);
        md.standard = M.type == FL_MAT_STANDARD ? M.standard : 0;
        md.texture = M.type == FL_MAT_LAMBERT ? M.texture - 1 : -1;
        s->materials_host.push_back(md);
    }
    const uint32_t n_std = d->standard_surfaces ? d->n_standard_surfaces : 0;
    std::vector<StandardDev> std_host;
    for (uint32_t i = 0; i < n_std; ++i) {
        std_host.push_back(standard_dev(d->standard_surfaces[i]));
        std_host.back().kd_texture = d->standard_surfaces[i].kd_texture - 1;
        std_host.back().bump_texture = d->standard_surfaces[i].bump_texture - 1;
    }
    s->n_standard = n_std;
    s->ext_kernels = n_std > 0;
    for (const MaterialDev &md : s->materials_host) s->ext_kernels |= md.texture >= 0;
    s->n_lights = d->n_lights;
    s->n_materials = d->n_materials;

    auto fail = [&](fl_status rc) {
        scene_release(s);  // ctx->mu is held
        return rc;
    };
    cudaError_t e;
#define SC_TRY(call)                                            \
    do {                                                        \
        e = (call);                                             \
        if (e != cudaSuccess) return fail(cuda_status(ctx, e, #call)); \
    } while (0)
#define SC_TRY_RC(call)                                         \
    do {                                                        \
        const fl_status r_ = (call);                            \
        if (r_ != FL_OK) return fail(r_);                       \
    } while (0)
    SC_TRY(cudaSetDevice(ctx->device));
    const size_t nt = d->n_tri ? d->n_tri : 1;
    SC_TRY_RC(dev_alloc_n(ctx, &s->soup, 9 * nt));
    SC_TRY_RC(dev_alloc_n(ctx, &s->tri_material, nt));
    SC_TRY_RC(dev_alloc_n(ctx, &s->tri_light, nt));
    SC_TRY_RC(dev_alloc_n(ctx, &s->materials, d->n_materials));
    SC_TRY_RC(dev_alloc_n(ctx, &s->lights, d->n_lights));
    SC_TRY_RC(dev_alloc_n(ctx, &s->mat_refl60, 60 * (size_t)d->n_materials));
    {
        // from_reflectance_rgb (color/spectrumoperations.cpp:113-147) over the 60 bins
        std::vector<float> refl((size_t)60 * d->n_materials);
        for (uint32_t m = 0; m < d->n_materials; ++m)
            refl60(ctx->binned_host, s->materials_host[m].basis, s->materials_host[m].w, &refl[(size_t)m * 60]);
        SC_TRY(cudaMemcpyAsync(s->mat_refl60, refl.data(), sizeof(float) * refl.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (d->uvs && d->n_tri) {
        SC_TRY_RC(dev_alloc_n(ctx, &s->uvs, 6 * (size_t)d->n_tri));
        SC_TRY(cudaMemcpyAsync(s->uvs, d->uvs, sizeof(float) * 6 * (size_t)d->n_tri, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (d->images && d->n_images) {
        std::vector<ImageDev> info(d->n_images);
        unsigned long long total = 0;
        for (uint32_t i = 0; i < d->n_images; ++i) {
            info[i] = ImageDev{total, d->images[i].width, d->images[i].height};
            total += 3ull * (unsigned long long)d->images[i].width * (unsigned long long)d->images[i].height;
        }
        SC_TRY_RC(dev_alloc_n(ctx, &s->pixels, total));
        SC_TRY_RC(dev_alloc_n(ctx, &s->images, d->n_images));
        for (uint32_t i = 0; i < d->n_images; ++i)
            SC_TRY(cudaMemcpyAsync(s->pixels + info[i].offset, d->images[i].rgb,
                                   3ull * (unsigned long long)d->images[i].width * (unsigned long long)d->images[i].height,
                                   cudaMemcpyHostToDevice, ctx->stream));
        SC_TRY(cudaMemcpyAsync(s->images, info.data(), sizeof(ImageDev) * d->n_images, cudaMemcpyHostToDevice,
                               ctx->stream));
        s->n_images = d->n_images;
    }
    SC_TRY_RC(dev_alloc_n(ctx, &s->standard, n_std));
    const size_t std_floats = (size_t)kStdSpectra * 60;
    SC_TRY_RC(dev_alloc_n(ctx, &s->std_refl60, std_floats * (n_std ? n_std : 1)));
    if (n_std) {
        std::vector<float> refl(std_floats * n_std);
        for (uint32_t m = 0; m < n_std; ++m) {
            float *row = &refl[(size_t)m * std_floats];
            for (int c = 0; c < 5; ++c) refl60(ctx->binned_host, std_host[m].basis[c], std_host[m].w[c], row + 60 * c);
            // GetMetalCoefficientsFromForge (color/metallurgy.cpp:42-74): unknown types are gold
            const int mt = d->standard_surfaces[m].metal_type;
            const int metal = (mt >= 0 && mt <= 8) ? mt : 0;
            std::memcpy(row + 300, &ctx->metal60[120 * (size_t)metal], sizeof(float) * 120);
        }
        SC_TRY(cudaMemcpyAsync(s->standard, std_host.data(), sizeof(StandardDev) * n_std, cudaMemcpyHostToDevice,
                               ctx->stream));
        SC_TRY(cudaMemcpyAsync(s->std_refl60, refl.data(), sizeof(float) * refl.size(), cudaMemcpyHostToDevice,
                               ctx->stream));
    }
    if (d->n_tri) {
        SC_TRY(cudaMemcpyAsync(s->soup, d->verts, sizeof(float) * 9 * d->n_tri, cudaMemcpyHostToDevice, ctx->stream));
        if (d->tri_material)
            SC_TRY(cudaMemcpyAsync(s->tri_material, d->tri_material, sizeof(uint32_t) * d->n_tri,
                                   cudaMemcpyHostToDevice, ctx->stream));
        else
            SC_TRY(cudaMemsetAsync(s->tri_material, 0, sizeof(uint32_t) * d->n_tri, ctx->stream));
        // no triangle emits but the lights' own (set on the device below)
        SC_TRY(cudaMemsetAsync(s->tri_light, 0xff, sizeof(int32_t) * d->n_tri, ctx->stream));
    }
    SC_TRY(cudaMemcpyAsync(s->materials, s->materials_host.data(), sizeof(MaterialDev) * d->n_materials,
                           cudaMemcpyHostToDevice, ctx->stream));
    if (d->n_lights) {
        SC_TRY(cudaMemcpyAsync(s->lights, lights_dev.data(), sizeof(LightDev) * d->n_lights, cudaMemcpyHostToDevice,
                               ctx->stream));
        if (s->n_emissive_tris) {
            k_tri_light<<<(d->n_lights + 127) / 128, 128, 0, ctx->stream>>>(s->lights, d->n_lights, s->tri_light);
            SC_TRY(cudaGetLastError());
        }
    }
#undef SC_TRY
#undef SC_TRY_RC
    fl_status rc = build_bvh(s);
    if (rc != FL_OK) return fail(rc);
    ctx->children++;
    s->counted = true;
    *out = reinterpret_cast<fl_scene *>(s);
    return FL_OK;
}

fl_status fl_scene_destroy(fl_scene *scene) {
    Scene *s = reinterpret_cast<Scene *>(scene);
    if (!s) return FL_ERR_INVALID;
    // The context's lock: its stream may be capturing a render's graph on another thread,
    // and neither the synchronisation nor the frees may enter that capture.
    std::lock_guard<std::mutex> lock(s->ctx->mu);
    scene_release(s);
    return FL_OK;
}

fl_status fl_scene_get_info(const fl_scene *scene, fl_scene_info *info) {
    const Scene *s = reinterpret_cast<const Scene *>(scene);
    if (!s || !info) return FL_ERR_INVALID;
    info->n_tri = s->n_tri;
    info->n_nodes = s->n_nodes;
    info->n_leaves = s->n_leaves;
    info->max_depth = s->max_depth;
    info->bvh_bytes = (uint64_t)s->n_nodes * sizeof(WideNode) + (uint64_t)s->n_tri * 48u;
    info->build_ms = s->build_ms;
    return FL_OK;
}

}  // extern "C"
