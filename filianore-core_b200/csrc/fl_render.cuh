// Wavefront path tracer: the GPU replacement of the absent application's loop over
// pixels and samples that calls PathIntegrator::Li
// (src/filianore/integrators/pathintegrator.cpp:12-87) with estimate_direct
// (src/filianore/integrators/integrator.cpp:25-110) for every light.
//
// A wave holds up to `cap` camera samples. Per bounce, four kernels run over SoA queues:
//   k_trace_paths  closest hit of every live path ray (8-wide BVH + analytic sphere lights)
//   k_shade        emission, miss handling, and for every light the two NEE candidates
//                  of estimate_direct (light sample -> shadow ray; BSDF sample -> MIS ray),
//                  fully weighted; live paths are compacted into the continuation queue
//   k_trace_rays2  shadow rays (reference visibility rule) and MIS rays (did the BSDF
//                  sample reach this light?), one launch for both kinds
//   k_continue     adds the visible NEE terms in the reference's order, samples the
//                  continuation, applies depth cut-offs and Russian roulette, and
//                  compacts surviving paths into the next queue
// Random numbers are drawn in the reference's order (per light: uLight, uScatter; then
// the BSDF sample; then RR), so a path consumes its PCG32 stream exactly as
// PathIntegrator::Li does. Queues are compacted with warp ballots and one atomic per warp.
// Kernels read their item counts from device memory, so a whole wave is enqueued without
// host synchronisation. Finished paths add to_xyz(L) to an FP64 film with atomics.
#pragma once

#include <cstddef>
#include <vector>

#include "fl_guide.cuh"
#include "fl_internal.h"
#include "fl_shading.cuh"
#include "fl_traverse.cuh"

namespace fl {

// 0: miss, 1 + material type (Lambert, conductor, rough / smooth dielectric, standard
// surface; image-textured Lambert joins the standard surfaces), and with guiding on,
// kClassLambertLate: Lambert vertices past the guided ones (no inference)
constexpr int kShadeClasses = 7;
constexpr int kClassStandard = 1 + FL_MAT_STANDARD;
constexpr int kClassLambertLate = 6;
static_assert(1 + FL_MAT_STANDARD < kClassLambertLate, "one shading class per material type");
constexpr int kGuidedVertices = 2;  // a path's first Lambert vertices are guided (and recorded)
// path flags: bits 0..7 bounce, bit 8 specular, bits 9..10 Lambert vertices passed (guiding)
__device__ __forceinline__ uint32_t lambert_count(uint32_t fl) { return (fl >> 9) & 3u; }
constexpr int kMaxJobs = 64;      // jobs that can share one wave (serving)
constexpr int kMaxSegs = 128;     // sample ranges per wave

struct WaveCounters {
    uint32_t n_trace, n_cont, n_next, n_shadow;
    uint32_t fetch_trace, fetch_rays2;              // persistent-kernel work counters
    uint32_t n_cont_std, pad1;                      // StandardSurface paths, from the back of q_cont
    uint32_t n_class[8];                            // shading queues by class
    unsigned long long rays, shadow_rays, bounces, paths;
    unsigned long long nodes, tris;  // FL_RENDER_COUNT
    int err;
    uint32_t cut;                    // paths ended at the job's bounce cap
    // streaming waves (path regeneration): free path slots, paths of the wave started so
    // far, and this iteration's new paths (the regen_n lowest free slots take wave paths
    // regen_base, +regen_n and are queued at q_trace[regen_dst, +regen_n))
    uint32_t n_free, next_path;
    uint32_t regen_n, regen_dst, regen_base, pad3;
};

// FL_RENDER_PROFILE: CUDA events bracketing every launch, grouped by kernel class. The
// events come from a pool owned by the context and are reused by later renders.
struct RenderProfile {
    bool on = false;
    std::vector<cudaEvent_t> *pool = nullptr;
    size_t used = 0;
    std::vector<cudaEvent_t> ev[4];  // pairs (start, stop) per class: trace, shade, shadow, continue
    uint32_t launches = 0;
    void mark(int cls, cudaStream_t st) {
        if (!on || !pool) return;
        if (used == pool->size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) {
                on = false;
                return;
            }
            pool->push_back(e);
        }
        cudaEvent_t e = (*pool)[used++];
        cudaEventRecord(e, st);
        ev[cls].push_back(e);
    }
    void sum(double ms[4]) {
        for (int c = 0; c < 4; ++c) {
            ms[c] = 0.0;
            for (size_t i = 0; i + 1 < ev[c].size(); i += 2) {
                float t = 0.f;
                cudaEventElapsedTime(&t, ev[c][i], ev[c][i + 1]);
                ms[c] += t;
            }
        }
    }
};

struct CamDev {
    v3 origin, lower_left, horizontal, vertical, u, v;
    int W, H;
    float lens_radius;  // PhysicalCamera::lensRadius = aperture / 2 (0: pinhole)
};

// fl_li: a batch of caller rays in place of the camera's. Ray i is "pixel" i of a 1-spp
// job; it starts from the caller's PCG32 state (increment 3) and hero wavelength, and its
// radiance spectrum and final generator state are written back.
struct LiRays {
    const float4 *org, *dir;            // (o, tmin), (d, tmax)
    const unsigned long long *rng;      // PCG32 state per ray
    const float *lambda0;               // hero wavelength per ray (hero mode)
    float *L;                           // NL floats per ray
    unsigned long long *rng_out;        // generator state when the path ended (nullable)
};

// Everything one render job needs: its scene, camera, parameters and film. A wave's paths
// may belong to different jobs (serving); every kernel looks its path's job up.
struct JobDev {
    const WideNode *nodes;
    uint32_t n_nodes;
    const float4 *tris;
    uint32_t n_tri;
    const float *soup;
    const uint32_t *tri_material;
    const int32_t *tri_light;
    const MaterialDev *materials;
    const float *mat_refl60;
    const StandardDev *standard;
    const float *std_refl60;
    const float *uvs;              // 6 per triangle, or null
    const unsigned char *pixels;   // image bytes
    const ImageDev *images;
    const LightDev *lights;
    int n_lights;
    int any_hit_ok;
    int has_env;
    int has_spheres;
    float env_radiance;
    CamDev cam;
    int spp;
    int depth[3];       // RenderParams: diffuse, reflection (specular + glossy), transmission
    int bounce_cap;     // paths alive after bounce bounce_cap - 1 are cut (FL_MAX_BOUNCES)
    float rr_threshold;
    uint32_t sample_offset;
    uint32_t n_pix;
    double *film;  // FP64 XYZ sums, 3 per pixel
    int corrected_ggx;  // FL_RENDER_CORRECTED_GGX
    LiRays li;          // fl_li batches (li.org == nullptr for camera jobs)
};

// A wave is a list of sample ranges: slots [slot_begin, slot_begin + count) render the
// job's samples [sample_base, sample_base + count) in pixel-major order
// (sample index = g / n_pix, pixel = g % n_pix).
struct WaveSeg {
    uint32_t job, slot_begin, count, pad;
    unsigned long long sample_base, pad2;
};
struct WaveDesc {
    uint32_t n_wave, n_seg, pad[2];
    WaveSeg seg[kMaxSegs];
};

// A path's scalar state in one 32-byte record, so that a shading kernel, which visits
// slots in material order, reads it from one sector.
struct alignas(32) PathHead {
    unsigned long long rng;  // PCG32 state (increment 3)
    float lambda0;           // hero wavelength
    uint32_t flags;          // bits 0..7 bounce, bit 8 specular, bits 9..10 Lambert vertices (guiding)
    uint32_t pixel;
    uint32_t job;
    float eta_scale;
    uint32_t pad;
};
static_assert(sizeof(PathHead) == 32, "one sector per path");

struct RenderArgs {
    TablesArg tab;
    const JobDev *jobs;      // device, kMaxJobs entries
    const JobDev *job0;      // &jobs[0] when every path of the wave belongs to job 0 (no per-path lookup), else null
    const WaveDesc *wave;    // device
    int nl;                  // pending-term slots per path: the most lights of any job
    uint32_t cap;            // paths per wave
    // path state, slot-indexed; a slot's spectra are contiguous: x[slot * NL + k]
    PathHead *head;
    float *beta, *L;
    float4 *ray_o, *ray_d;
    int4 *hit;
    // pending NEE terms: C*[(li * cap + slot) * NL + k], pflags[li * cap + slot]
    float *CL, *CS;
    uint32_t *pflags;
    // shadow / MIS rays
    float4 *sray_o, *sray_d;
    uint32_t *stag;
    uint32_t scap;
    // queues
    uint32_t *q_trace, *q_cont, *q_next;
    uint32_t *q_class;  // kShadeClasses x cap: traced paths grouped by what shades them
    // streaming waves (null for fixed waves): 1 marks a slot whose path has ended, and per
    // chunk of kFreeChunk slots their count and the exclusive prefix of the counts
    uint8_t *slot_free;
    uint32_t *free_count, *free_off;
    unsigned long long *job_done;  // streaming server: finished paths per job table entry (else null)
    WaveCounters *cnt;
    GuideArgs g;        // learned guiding (zero when off)
};

enum : uint32_t { kHasCL = 1u, kHasCS = 2u, kVisOK = 4u, kMisOK = 8u };

// A shadow / MIS ray's tag: its path slot (< 2^25), light (< 64) and kind (0 shadow, 1 MIS)
constexpr uint32_t kMaxWaveSlots = 1u << 25;
__device__ __forceinline__ uint32_t shadow_tag(uint32_t slot, uint32_t li, uint32_t kind) {
    return (slot << 7) | (li << 1) | kind;
}

// queue append from divergent code: one atomic per group of converged lanes
__device__ inline uint32_t coalesced_append(uint32_t *counter, bool pred) {
    const uint32_t active = __activemask();
    const uint32_t mask = __ballot_sync(active, pred);
    if (!pred) return 0;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// append to one of several queues from divergent code: lanes with the same class share an atomic
__device__ inline uint32_t coalesced_append_class(uint32_t *counters, int cls) {
    const uint32_t active = __activemask();
    const uint32_t same = __match_any_sync(active, cls);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(same) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&counters[cls], (uint32_t)__popc(same));
    base = __shfl_sync(same, base, leader);
    return base + __popc(same & ((1u << lane) - 1u));
}

// warp-aggregated queue append: returns this lane's position (valid when pred)
__device__ inline uint32_t warp_append(uint32_t *counter, bool pred) {
    const uint32_t mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return 0;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ inline void warp_count(unsigned long long *dst, uint32_t v) {
    unsigned long long x = v;
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(dst, x);
}

__device__ inline uint32_t load_count(const uint32_t *p) { return *(volatile const uint32_t *)p; }

// grid-stride loop whose trip count is uniform within a warp (for the warp collectives)
#define FL_WARP_UNIFORM_LOOP(i, n)                                                              \
    for (uint32_t _base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u,                       \
                  _stride = gridDim.x * blockDim.x, i = _base + (threadIdx.x & 31);             \
         _base < (n); _base += _stride, i = _base + (threadIdx.x & 31))

template <int NL>
__device__ inline void load_spec(const float *a, uint32_t cap, uint32_t slot, Spec<NL> &s) {
    // a slot's NL samples are contiguous (16-byte aligned): the shading kernels visit slots
    // in material order, so one path's spectrum is one or a few sectors, not NL of them
    static_assert(NL % 4 == 0, "spectra are stored as float4 groups");
    (void)cap;
    const float4 *p = reinterpret_cast<const float4 *>(a + (size_t)slot * NL);
#pragma unroll
    for (int k = 0; k < NL / 4; ++k) {
        const float4 v = p[k];
        s.c[4 * k] = v.x; s.c[4 * k + 1] = v.y; s.c[4 * k + 2] = v.z; s.c[4 * k + 3] = v.w;
    }
}
template <int NL>
__device__ inline void store_spec(float *a, uint32_t cap, uint32_t slot, const Spec<NL> &s) {
    (void)cap;
    float4 *p = reinterpret_cast<float4 *>(a + (size_t)slot * NL);
#pragma unroll
    for (int k = 0; k < NL / 4; ++k) p[k] = make_float4(s.c[4 * k], s.c[4 * k + 1], s.c[4 * k + 2], s.c[4 * k + 3]);
}

template <int NL>
__device__ inline void finish_path(const RenderArgs &A, const JobDev &J, const SmemTables &sm, uint32_t slot,
                                   const Spec<NL> &L) {
    double xyz[3];
    spectrum_xyz<NL>(sm, A.tab, A.head[slot].lambda0, L, xyz);
    const uint32_t pix = A.head[slot].pixel;
    if (A.slot_free) A.slot_free[slot] = 1;  // streaming: the slot takes a new path
    if (A.job_done) {  // one atomic per job among the converged lanes
        const uint32_t job = A.head[slot].job;
        const uint32_t peers = __match_any_sync(__activemask(), job);
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&A.job_done[job], (unsigned long long)__popc(peers));
    }
    atomicAdd(&J.film[3 * (size_t)pix + 0], xyz[0]);
    atomicAdd(&J.film[3 * (size_t)pix + 1], xyz[1]);
    atomicAdd(&J.film[3 * (size_t)pix + 2], xyz[2]);
    if (J.li.L) {
        // Integrator::Li's return value and the sampler's state after the path
        store_spec<NL>(J.li.L, 0, pix, L);
        if (J.li.rng_out) J.li.rng_out[pix] = A.head[slot].rng;
    }
    if constexpr (NL == 4) {
        // guiding: the radiance gathered after each recorded vertex, divided by the
        // throughput it was scaled by, estimates the incident radiance along the
        // recorded direction (averaged over the hero wavelengths that carry any)
        if (A.g.rec_idx) {
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const uint32_t idx = A.g.rec_idx[(size_t)r * A.cap + slot];
                if (idx == kNoRecord) continue;
                float *R = A.g.rec + (size_t)idx * kRecFloats;
                float li = 0.f;
                int nz = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float b = R[12 + k];
                    if (b > 0.f) {
                        li += fmaxf(L.c[k] - R[16 + k], 0.f) / b;
                        ++nz;
                    }
                }
                R[11] = nz ? li / (float)nz : 0.f;
            }
        }
    }
}

// the hit record of BVH::intersect (bvh.cpp:49-84): p = o + d t, n = normalize(Ng), wo = normalize(-d)
__device__ inline Hit make_hit(const JobDev &A, float4 o4, float4 d4, int4 h) {
    Hit r;
    const v3 o = mk(o4.x, o4.y, o4.z), d = mk(d4.x, d4.y, d4.z);
    const float t = __int_as_float(h.y);
    r.p = add(o, mul(d, t));
    r.wo = normalize(neg(d));
    r.prim = h.x;
    r.b1 = __int_as_float(h.z);
    r.b2 = __int_as_float(h.w);
    if (h.x >= 0) {
        const v3 v0 = tri_v(A.soup, (uint32_t)h.x, 0), v1 = tri_v(A.soup, (uint32_t)h.x, 1),
                 v2 = tri_v(A.soup, (uint32_t)h.x, 2);
        r.n = normalize(cross(sub(v1, v0), sub(v2, v0)));
    } else {
        const LightDev &L = A.lights[-2 - h.x];
        r.n = normalize(sub(r.p, mk(L.cx, L.cy, L.cz)));
    }
    return r;
}

__device__ inline int prim_light(const JobDev &A, int prim) {
    if (prim >= 0) return A.tri_light[prim];
    if (prim <= -2) return -2 - prim;
    return -1;
}

// The hit's texture coordinates uv0 (1 - b1 - b2) + uv1 b1 + uv2 b2, each operation rounded
// on its own in both builds; (0, 0) without uvs, as BVH::intersect (bvh/bvh.cpp:69-71) leaves them.
__device__ inline void hit_uv(const JobDev &A, const Hit &h, float &u, float &v) {
    u = v = 0.f;
    if (!A.uvs || h.prim < 0) return;
    const float *t = A.uvs + 6 * (size_t)h.prim;
    const float w = __fsub_rn(__fsub_rn(1.f, h.b1), h.b2);
    u = __fadd_rn(__fadd_rn(__fmul_rn(__ldg(t + 0), w), __fmul_rn(__ldg(t + 2), h.b1)), __fmul_rn(__ldg(t + 4), h.b2));
    v = __fadd_rn(__fadd_rn(__fmul_rn(__ldg(t + 1), w), __fmul_rn(__ldg(t + 3), h.b1)), __fmul_rn(__ldg(t + 5), h.b2));
}

// ImageMapTexture::evaluate (shading/textures/imagemap.cpp:36-62): the nearest texel, then
// from_reflectance_rgb of it / 255, at the path's spectral samples. For j past the last row
// the reference sets i = height - 1 and reads outside the image; here j is clamped too.
__device__ inline const unsigned char *image_texel(const JobDev &A, int img, float u, float v) {
    const ImageDev im = A.images[img];
    int i = (int)__fmul_rn(u, (float)im.width);
    int j = (int)__fsub_rn(__fmul_rn(__fsub_rn(1.f, v), (float)im.height), 0.001f);
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > im.width - 1) i = im.width - 1;
    if (j > im.height - 1) { i = im.height - 1; j = im.height - 1; }
    if (i > im.width - 1) i = im.width - 1;
    return A.pixels + im.offset + 3ull * ((unsigned long long)j * (unsigned)im.width + (unsigned)i);
}

template <int NL>
__device__ inline void image_reflectance(const JobDev &A, const TablesArg &tab, const SmemTables &sm, int img, float u,
                                         float v, float lambda0, Spec<NL> &out) {
    const unsigned char *px = image_texel(A, img, u, v);
    const float rgb[3] = {(float)(int)px[0] / 255.f, (float)(int)px[1] / 255.f, (float)(int)px[2] / 255.f};
    int basis[3];
    float w[3];
    smits_terms(rgb, basis, w);
    for (int k = 0; k < NL; ++k) {
        if (NL == 60) {
            float r = 0.f;
            for (int q = 0; q < 3; ++q) r += sm.binned[180 + 60 * basis[q] + k] * w[q];
            r *= 0.94f;
            out.c[k] = r < 0.f ? 0.f : r;
        } else {
            out.c[k] = smits_at(sm, tab, basis, w, hero_lambda(lambda0, k));
        }
    }
}

// Material::bump_evaluate (materials/material.cpp:8-31) with the bump map's red channel as
// height: the shading normal of a hit on triangle h.prim. dpdu, dpdv follow
// Triangle::intersect (shapes/triangle.cpp:33-52) over the vertex uvs (all zero without uvs).
static __device__ __noinline__ v3 bump_normal(const JobDev &A, const Hit &h, int img) {
    const v3 p1 = tri_v(A.soup, (uint32_t)h.prim, 0), p2 = tri_v(A.soup, (uint32_t)h.prim, 1),
             p3 = tri_v(A.soup, (uint32_t)h.prim, 2);
    float uv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (A.uvs)
        for (int k = 0; k < 6; ++k) uv[k] = __ldg(A.uvs + 6 * (size_t)h.prim + k);
    const float duv02x = __fsub_rn(uv[0], uv[4]), duv02y = __fsub_rn(uv[1], uv[5]);
    const float duv12x = __fsub_rn(uv[2], uv[4]), duv12y = __fsub_rn(uv[3], uv[5]);
    const v3 dp02 = sub(p1, p3), dp12 = sub(p2, p3);
    const float determinant = __fsub_rn(__fmul_rn(duv02x, duv12y), __fmul_rn(duv02y, duv12x));
    const bool degenerate = fabs((double)determinant) < 1e-8;
    v3 dpdu = mk(0.f, 0.f, 0.f), dpdv = mk(0.f, 0.f, 0.f);
    if (!degenerate) {
        const float invDet = __fdiv_rn(1.f, determinant);
        dpdu = mul(sub(mul(dp02, duv12y), mul(dp12, duv02y)), invDet);
        dpdv = mul(add(mul(dp02, -duv12x), mul(dp12, duv02x)), invDet);
    }
    if (degenerate || len2(cross(dpdu, dpdv)) == 0.f) coordinate_system(cross(sub(p2, p1), sub(p3, p1)), &dpdu, &dpdv);
    float u, v;
    hit_uv(A, h, u, v);
    const float du = 0.0005f, dv = 0.0005f;
    const float uDisplace = (float)(int)image_texel(A, img, __fadd_rn(u, du), v)[0] / 255.f;
    const float vDisplace = (float)(int)image_texel(A, img, u, __fadd_rn(v, dv))[0] / 255.f;
    const float displace = (float)(int)image_texel(A, img, u, v)[0] / 255.f;
    const v3 bu = add(dpdu, mul(mul(h.n, __fdiv_rn(__fsub_rn(uDisplace, displace), du)), 4.f));
    const v3 bv = add(dpdv, mul(mul(h.n, __fdiv_rn(__fsub_rn(vDisplace, displace), dv)), 4.f));
    // set_shading_geometry (core/interaction.cpp:20-33): normal of (bu, bv) on n's side
    const v3 ns = normalize(cross(bu, bv));
    return dot(ns, h.n) < 0.f ? neg(ns) : ns;
}

template <int NL, bool STD>
__device__ inline void make_bsdf(const JobDev &A, const TablesArg &tab, const SmemTables &sm, const Hit &h,
                                 float lambda0, Bsdf<NL> &b) {
    b.ng = h.n;
    b.ns = h.n;
    coordinate_system(b.ns, &b.s, &b.t);
    b.s = normalize(b.s);
    const uint32_t mi = h.prim >= 0 ? A.tri_material[h.prim] : 0u;
    const MaterialDev m = A.materials[mi];
    b.type = m.type;
    b.mat_eta = m.eta;
    b.mat_k = m.k;
    b.ax = m.ax;
    b.ay = m.ay;
    b.eta = (m.type == FL_MAT_ROUGH_DIELECTRIC || m.type == FL_MAT_SMOOTH_DIELECTRIC) ? m.eta : 1.f;
    b.corrected = A.corrected_ggx;
    if (STD && m.type == FL_MAT_LAMBERT) {
        // LambertMaterial with an ImageMapTexture (materials/lambert.cpp:8-15)
        float u, v;
        hit_uv(A, h, u, v);
        image_reflectance<NL>(A, tab, sm, m.texture, u, v, lambda0, b.R);
        return;
    }
    if (STD) {
        // StandardSurfaceMaterial::compute_scattering_functions (materials/standardsurface.cpp:72-159)
        // from the host-reduced record
        const StandardDev *sd = A.standard + m.standard;
        b.sd = sd;
        b.eta = sd->eta;
        b.mat_eta = sd->ior;
        b.ax = sd->ax;
        b.ay = sd->ay;
        b.std60 = A.std_refl60 + kStdSpectra * 60 * (size_t)m.standard;
        b.bases = sm.bases;
        b.rgb_l0 = tab.rgb_lambda0;
        b.rgb_l1 = tab.rgb_lambda1;
        b.n_rgb = tab.n_rgb;
        b.lambda0 = lambda0;
        b.kd_tex = sd->kd_texture >= 0;
        if (sd->bump_texture >= 0 && h.prim >= 0) {
            b.ns = bump_normal(A, h, sd->bump_texture);
            coordinate_system(b.ns, &b.s, &b.t);
            b.s = normalize(b.s);
        }
        if (b.kd_tex) {
            float u, v;
            hit_uv(A, h, u, v);
            image_reflectance<NL>(A, tab, sm, sd->kd_texture, u, v, lambda0, b.R);
        }
        return;
    }
    if (m.type == FL_MAT_LAMBERT) {
        reflectance<NL>(sm, tab, m, A.mat_refl60 + 60 * (size_t)mi, lambda0, b.R);
    } else {
        b.R.set(1.f);
    }
}

// ------------------------------------------------------------------------------ kernels

// Starts path q of the wave (its segment gives the job and the sample index) in slot k: the
// camera ray (or fl_li's ray) and the initial path state. The caller queues the slot.
template <int NL>
__device__ inline void init_path(const RenderArgs &A, uint32_t k, uint32_t q) {
    const uint32_t n_seg = A.wave->n_seg;
    uint32_t si = 0;
    while (si + 1 < n_seg && q >= A.wave->seg[si + 1].slot_begin) ++si;
    const WaveSeg sg = A.wave->seg[si];
    const JobDev &J = A.jobs[sg.job];
    const unsigned long long g = sg.sample_base + (q - sg.slot_begin);
    const uint32_t pix = (uint32_t)(g % J.n_pix);
    const unsigned long long s = g / J.n_pix;
    if (J.li.org) {
        // fl_li: the caller's ray, generator state and wavelength
        PathHead ph;
        ph.rng = J.li.rng[pix];
        ph.lambda0 = J.li.lambda0 ? J.li.lambda0[pix] : 380.f;
        ph.flags = 0u;
        ph.pixel = pix;
        ph.job = sg.job;
        ph.eta_scale = 1.f;
        ph.pad = 0u;
        A.head[k] = ph;
        Spec<NL> one, zero;
        one.set(1.f);
        zero.set(0.f);
        store_spec<NL>(A.beta, A.cap, k, one);
        store_spec<NL>(A.L, A.cap, k, zero);
        A.ray_o[k] = J.li.org[pix];
        A.ray_d[k] = J.li.dir[pix];
        if (A.g.rec_idx) {
            A.g.rec_idx[k] = kNoRecord;
            A.g.rec_idx[(size_t)A.cap + k] = kNoRecord;
        }
        return;
    }
    Pcg32 rng;
    rng.seed(pix, 1u);
    const unsigned long long sidx = (unsigned long long)J.sample_offset + s;
    if (sidx) rng.advance(sidx << 16);
    const float ux = rng.nextf(), uy = rng.nextf(), ul = rng.nextf();
    const uint32_t px = pix % (uint32_t)J.cam.W, py = pix / (uint32_t)J.cam.W;
    const float sx = __fdiv_rn(__fadd_rn((float)px, ux), (float)J.cam.W);
    const float sy = __fdiv_rn(__fadd_rn((float)((uint32_t)J.cam.H - 1u - py), uy), (float)J.cam.H);
    // PhysicalCamera::awaken_ray (cameras/physical.cpp:12-22): a pinhole takes the lens
    // sample (0.5, 0.5); a lens draws two numbers and maps them with the concentric disk
    v3 rd;
    if (J.cam.lens_radius > 0.f) {
        const float lx = rng.nextf(), ly = rng.nextf();
        const v3 lp = concentric_disk(lx, ly);
        rd = mul(lp, J.cam.lens_radius);
    } else {
        const v3 lp = sub(mul(mk(0.5f, 0.5f, 0.f), 2.f), mk(1.f, 1.f, 0.f));
        rd = mul(lp, 0.f);
    }
    const v3 offset = add(mul(J.cam.u, rd.x), mul(J.cam.v, rd.y));
    const v3 o = add(J.cam.origin, offset);
    const v3 dir = sub(sub(add(add(J.cam.lower_left, mul(J.cam.horizontal, sx)), mul(J.cam.vertical, sy)),
                           J.cam.origin),
                       offset);
    const v3 d = normalize(dir);
    PathHead ph;
    ph.rng = rng.state;
    ph.lambda0 = __fadd_rn(380.f, __fmul_rn(ul, 340.f));  // not contracted: the oracle rounds twice
    ph.flags = 0u;
    ph.pixel = pix;
    ph.job = sg.job;
    ph.eta_scale = 1.f;
    ph.pad = 0u;
    A.head[k] = ph;
    Spec<NL> one, zero;
    one.set(1.f);
    zero.set(0.f);
    store_spec<NL>(A.beta, A.cap, k, one);
    store_spec<NL>(A.L, A.cap, k, zero);
    A.ray_o[k] = make_float4(o.x, o.y, o.z, 0.f);
    A.ray_d[k] = make_float4(d.x, d.y, d.z, __int_as_float(0x7f800000));
    if (A.g.rec_idx) {
        A.g.rec_idx[k] = kNoRecord;
        A.g.rec_idx[(size_t)A.cap + k] = kNoRecord;
    }
}

template <int NL>
__global__ void __launch_bounds__(128) k_raygen(RenderArgs A) {
    const uint32_t n_wave = A.wave->n_wave;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.cnt->n_trace = n_wave;
        A.cnt->n_cont = A.cnt->n_next = A.cnt->n_shadow = A.cnt->n_cont_std = 0;
        A.cnt->fetch_trace = A.cnt->fetch_rays2 = 0;
        for (int c = 0; c < kShadeClasses; ++c) A.cnt->n_class[c] = 0;
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_wave; k += gridDim.x * blockDim.x) {
        init_path<NL>(A, k, k);
        A.q_trace[k] = k;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&A.cnt->paths, (unsigned long long)n_wave);
}

// Streaming waves (path regeneration). The wave descriptor lists more paths than there are
// slots; a path that ends frees its slot (finish_path), and every iteration starts as many
// new paths as there are free slots, so the late bounces of early paths run alongside the
// first bounces of later ones and the slots stay full until the descriptor's paths run out.
// New paths take the lowest free slots in slot order, so the paths started together sit in
// neighbouring slots and the kernels read and write their state in whole sectors.
constexpr uint32_t kFreeChunk = 4096;      // slots per block of the free-slot scan
constexpr uint32_t kMaxFreeChunks = 8192;  // covers kMaxWaveSlots
__host__ __device__ inline uint32_t free_chunks(size_t cap) { return (uint32_t)((cap + kFreeChunk - 1) / kFreeChunk); }

static __global__ void __launch_bounds__(128) k_stream_init(RenderArgs A) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.cap; i += gridDim.x * blockDim.x)
        A.slot_free[i] = 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        WaveCounters *c = A.cnt;
        c->n_free = A.cap;
        c->next_path = 0;
        c->n_next = 0;
        c->n_trace = 0;
        c->regen_n = c->regen_dst = c->regen_base = 0;
    }
}

// Free slots per chunk (one block of 256 threads per chunk, 16 flags per thread).
static __global__ void __launch_bounds__(256) k_free_count(RenderArgs A) {
    const uint32_t c0 = blockIdx.x * kFreeChunk;
    uint32_t n = 0;
    for (uint32_t i = c0 + threadIdx.x; i < min(c0 + kFreeChunk, A.cap); i += 256) n += A.slot_free[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    __shared__ uint32_t w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < 8; ++k) t += w[k];
        A.free_count[blockIdx.x] = t;
    }
}

// Iteration start (one block of 1024 threads): the prefix of the chunk counts, then the
// survivors of the last iteration head this iteration's trace queue and new paths follow.
static __global__ void __launch_bounds__(1024) k_stream_step(RenderArgs A) {
    const uint32_t nc = free_chunks(A.cap);
    constexpr int kPer = kMaxFreeChunks / 1024;
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint32_t i = threadIdx.x * kPer + k;
        v[k] = i < nc ? A.free_count[i] : 0u;
        sum += v[k];
    }
    // exclusive scan of the per-thread sums over the block
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ uint32_t wsum[32];
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t x = wsum[lane], xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        wsum[lane] = xi - x;  // exclusive prefix of the warp sums
    }
    __syncthreads();
    uint32_t run = wsum[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint32_t i = threadIdx.x * kPer + k;
        if (i < nc) A.free_off[i] = run;
        run += v[k];
    }
    if (threadIdx.x == 1023) {
        WaveCounters *c = A.cnt;
        const uint32_t n_free = run;  // the total
        // every slot is free or holds a survivor (checked, so that a broken count can only
        // stop the wave early, never index outside the buffers)
        uint32_t surv = c->n_next;
        uint32_t avail = n_free;
        if (surv > A.cap || avail > A.cap - surv) {
            c->err += 1;
            surv = min(surv, A.cap);
            avail = min(avail, A.cap - surv);
        }
        const uint32_t n_wave = A.wave->n_wave;
        const uint32_t remaining = n_wave > c->next_path ? n_wave - c->next_path : 0u;
        const uint32_t nn = min(avail, remaining);
        c->n_free = n_free;
        c->regen_n = nn;
        c->regen_dst = surv;
        c->regen_base = c->next_path;
        c->next_path += nn;
        c->n_trace = surv + nn;
        c->n_next = 0;
        c->n_cont = 0;
        c->n_cont_std = 0;
        c->n_shadow = 0;
        c->fetch_trace = 0;
        c->fetch_rays2 = 0;
        for (int k = 0; k < kShadeClasses; ++k) c->n_class[k] = 0;
    }
}

// New paths into the regen_n lowest free slots (one block of 256 threads per chunk): the
// r-th free slot of the wave starts path regen_base + r and is queued at regen_dst + r.
template <int NL>
__global__ void __launch_bounds__(256) k_regen(RenderArgs A) {
    const uint32_t nn = load_count(&A.cnt->regen_n);
    const uint32_t off = A.free_off[blockIdx.x];
    if (off >= nn) return;  // every free slot of this chunk stays free
    const uint32_t dst = A.cnt->regen_dst, base = A.cnt->regen_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t wcnt[8];
    uint32_t rank0 = off;  // rank of the first free slot of the next 256 slots
    const uint32_t c0 = blockIdx.x * kFreeChunk, c1 = min(c0 + kFreeChunk, A.cap);
    for (uint32_t r0 = c0; r0 < c1 && rank0 < nn; r0 += 256) {
        const uint32_t slot = r0 + threadIdx.x;
        const bool fr = slot < c1 && A.slot_free[slot] != 0;
        const uint32_t m = __ballot_sync(0xffffffffu, fr);
        if (lane == 0) wcnt[warp] = __popc(m);
        __syncthreads();
        uint32_t before = 0, total = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            before += k < warp ? wcnt[k] : 0u;
            total += wcnt[k];
        }
        const uint32_t rank = rank0 + before + __popc(m & ((1u << lane) - 1u));
        if (fr && rank < nn) {
            A.slot_free[slot] = 0;
            init_path<NL>(A, slot, base + rank);
            A.q_trace[dst + rank] = slot;
        }
        rank0 += total;
        __syncthreads();  // wcnt is reused
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && nn) atomicAdd(&A.cnt->paths, (unsigned long long)nn);
}

static __global__ void __launch_bounds__(128) k_advance(WaveCounters *cnt) {
    cnt->n_trace = cnt->n_next;
    cnt->n_next = 0;
    cnt->n_cont = 0;
    cnt->n_cont_std = 0;
    cnt->n_shadow = 0;
    cnt->fetch_trace = 0;
    cnt->fetch_rays2 = 0;
    for (int c = 0; c < kShadeClasses; ++c) cnt->n_class[c] = 0;
}

// analytic sphere lights after the triangle traversal: closest of both
__device__ inline void add_spheres(const JobDev &A, const RayPre &r, TraceResult &res) {
    if (!A.has_spheres) return;
    const v3 o = mk(r.ox, r.oy, r.oz), d = mk(r.dx, r.dy, r.dz);
    float best = res.id >= 0 ? res.t : r.tmax;
    for (int l = 0; l < A.n_lights; ++l) {
        const LightDev L = A.lights[l];
        if (L.type != FL_LIGHT_SPHERE) continue;
        const float ts = sphere_hit(L, o, d, r.tmin, best);
        if (ts > 0.f && ts < best) {
            best = ts;
            res.id = -2 - l;
            res.t = ts;
            res.u = res.v = 0.f;
        }
    }
}

#ifndef FL_TRACE_STEPS
#define FL_TRACE_STEPS 8
#endif
constexpr int kRenderTraceSteps = FL_TRACE_STEPS;  // traversal steps between refills of finished lanes
// Resident blocks per SM the render's traversal kernels are compiled for (caps registers).
// With streaming waves every launch has a full queue, and more warps per SM pay: the
// 1,048,578-triangle frame measured 1,632 Mrays/s at 6 blocks, 1,670 at 7, 1,697 at 8 and
// 1,695 at 9 (A/B on one B200).
#ifndef FL_RENDER_TRACE_BLOCKS
#define FL_RENDER_TRACE_BLOCKS 8
#endif
constexpr int kRenderTraceBlocks = FL_RENDER_TRACE_BLOCKS;
#ifndef FL_RENDER_RAYS2_BLOCKS
#define FL_RENDER_RAYS2_BLOCKS 8
#endif
constexpr int kRenderRays2Blocks = FL_RENDER_RAYS2_BLOCKS;  // the same for the shadow / MIS ray kernel
// resident blocks per SM that k_shade and k_continue are compiled for (0: no bound)
#ifndef FL_RENDER_SHADE_BLOCKS
#define FL_RENDER_SHADE_BLOCKS 0
#endif
#ifndef FL_RENDER_CONT_BLOCKS
#define FL_RENDER_CONT_BLOCKS 0
#endif
#if FL_RENDER_SHADE_BLOCKS > 0
#define FL_SHADE_BOUNDS __launch_bounds__(128, FL_RENDER_SHADE_BLOCKS)
#else
#define FL_SHADE_BOUNDS __launch_bounds__(128)
#endif
#if FL_RENDER_CONT_BLOCKS > 0
#define FL_CONT_BOUNDS __launch_bounds__(128, FL_RENDER_CONT_BLOCKS)
#else
#define FL_CONT_BOUNDS __launch_bounds__(128)
#endif

struct PathTraceItem {
    const RenderArgs *A;
    const JobDev *J;
    const WideNode *nodes;
    uint32_t n_nodes;
    const float4 *tris;
    uint32_t n_tris;
    uint32_t slot;
    bool any_hit;
    RayPre ray;
    TravState st;
    __device__ void bind_job0() {  // every path in job 0: its scene once, not per ray
        J = A->job0;
        nodes = J->nodes;
        n_nodes = J->n_nodes;
        tris = J->tris;
        n_tris = J->n_tri;
    }
    __device__ bool begin(uint32_t q) {
        slot = A->q_trace[q];
        if (!A->job0) {
            J = &A->jobs[A->head[slot].job];
            nodes = J->nodes;
            n_nodes = J->n_nodes;
            tris = J->tris;
            n_tris = J->n_tri;
        }
        ray = ray_precompute(A->ray_o[slot], A->ray_d[slot]);
        trav_init(st, ray);
        return true;
    }
    __device__ void finish() {
        TraceResult res = st.res;
        add_spheres(*J, ray, res);
        A->hit[slot] = make_int4(res.id, __float_as_int(res.t), __float_as_int(res.u), __float_as_int(res.v));
        // group by shading work so that warps of k_shade / k_continue run one material's code
        int cls = 0;
        if (res.id != -1) {
            const uint32_t mi = res.id >= 0 ? J->tri_material[res.id] : 0u;
            const MaterialDev &m = J->materials[mi];
            cls = (m.type == FL_MAT_LAMBERT && m.texture >= 0) ? kClassStandard : 1 + m.type;
            if (cls == 1 + FL_MAT_LAMBERT && A->g.select > 0.f && lambert_count(A->head[slot].flags) >= kGuidedVertices)
                cls = kClassLambertLate;
        }
        const uint32_t pos = coalesced_append_class(A->cnt->n_class, cls);
        A->q_class[(size_t)cls * A->cap + pos] = slot;
    }
};

// camera and continuation rays: closest hit (persistent, lanes refilled as rays finish)
template <bool COUNT>
__global__ void __launch_bounds__(128, kRenderTraceBlocks) k_trace_paths(RenderArgs A) {
    const uint32_t n = load_count(&A.cnt->n_trace);
    bool err = false;
    TraceStats st;
    PathTraceItem it;
    it.A = &A;
    it.any_hit = false;
    if (A.job0) it.bind_job0();
    __shared__ uint2 stack[trav_stack_smem_bytes(128) / sizeof(uint2)];
    __shared__ uint4 top[kSmemNodeWords];
    const uint32_t n_top = trav_stage_top(top, A.job0 ? it.nodes : nullptr, A.job0 ? it.n_nodes : 0u);
    persistent_trace<kRenderTraceSteps, COUNT>(it, &A.cnt->fetch_trace, n, err, st, stack, top, n_top);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&A.cnt->rays, (unsigned long long)n);
    if (COUNT) {
        warp_count(&A.cnt->nodes, st.nodes);
        warp_count(&A.cnt->tris, st.tris);
    }
    if (err) atomicAdd(&A.cnt->err, 1);
}

// STD: the StandardSurface instance, over the StandardSurface class alone; the other
// instance takes every other class
template <int NL, bool STD = false>
__global__ void FL_SHADE_BOUNDS k_shade(RenderArgs A) {
    __shared__ SmemTables sm;
    stage_tables(sm, A.tab, NL != 60);
    uint32_t off[kShadeClasses + 1];
    off[0] = 0;
    for (int c = 0; c < kShadeClasses; ++c)
        off[c + 1] = off[c] + ((c == kClassStandard) == STD ? load_count(&A.cnt->n_class[c]) : 0u);
    const uint32_t n = off[kShadeClasses];
    uint32_t shaded = 0;
    FL_WARP_UNIFORM_LOOP(q, n) {
        const bool active = q < n;
        bool alive = false;
        uint32_t slot = 0;
        if (active) {
            int c = 0;
            while (q >= off[c + 1]) ++c;
            slot = A.q_class[(size_t)c * A.cap + (q - off[c])];
            const JobDev &J = A.jobs[A.head[slot].job];
            const int4 h = A.hit[slot];
            const uint32_t fl = A.head[slot].flags;
            const uint32_t bounce = fl & 0xffu;
            const bool specular = (fl >> 8) & 1u;
            const float4 o4 = A.ray_o[slot], d4 = A.ray_d[slot];
            Spec<NL> beta, L;
            load_spec<NL>(A.beta, A.cap, slot, beta);
            load_spec<NL>(A.L, A.cap, slot, L);
            const bool hit = h.x != -1;
            Hit hr;
            if (hit) hr = make_hit(J, o4, d4, h);
            if (bounce == 0 || specular) {
                if (hit) {
                    const int li = prim_light(J, h.x);
                    if (li >= 0) {
                        const LightDev Ll = J.lights[li];
                        const float le = dot(hr.n, mk(-d4.x, -d4.y, -d4.z)) > 0.f ? Ll.radiance : 0.f;
#pragma unroll
                        for (int c = 0; c < NL; ++c) L.c[c] += beta.c[c] * le;
                    }
                } else if (J.has_env) {
#pragma unroll
                    for (int c = 0; c < NL; ++c) L.c[c] += beta.c[c] * J.env_radiance;
                }
            }
            if (!hit) {
                finish_path<NL>(A, J, sm, slot, L);
            } else {
                ++shaded;
                alive = true;
                store_spec<NL>(A.L, A.cap, slot, L);
                const float lambda0 = A.head[slot].lambda0;
                Bsdf<NL> b;
                make_bsdf<NL, STD>(J, A.tab, sm, hr, lambda0, b);
                if (bsdf_num_components<STD>(b, kBsdfAll & ~kBsdfSpecular) > 0) {
                    Pcg32 rng;
                    rng.state = A.head[slot].rng;
                    rng.inc = 3u;
                    const int bsdfFlags = kBsdfAll & ~kBsdfSpecular;
                    for (int li = 0; li < J.n_lights; ++li) {
                        const float ulx = rng.nextf(), uly = rng.nextf();
                        const float usx = rng.nextf(), usy = rng.nextf();
                        const LightDev Ll = J.lights[li];
                        uint32_t pf = 0;
                        Spec<NL> CL, CS;
                        CL.set(0.f);
                        CS.set(0.f);
                        // light sampling term
                        float scatteringPdf = 0.f;
                        v3 wi = mk(0.f, 0.f, 0.f);
                        const LightSample ls = light_sample_li(Ll, J.soup, hr, ulx, uly);
                        float illumPdf = ls.pdf;
                        if (ls.vis_kind) wi = ls.wi;
                        if (ls.pdf > 0 && ls.radiance != 0.f) {
                            Spec<NL> f;
                            bsdf_eval<STD>(b, hr.wo, wi, bsdfFlags, f);
                            const float ad = absdot(wi, b.ns);
#pragma unroll
                            for (int c = 0; c < NL; ++c) f.c[c] *= ad;
                            scatteringPdf = bsdf_pdf<STD>(b, hr.wo, wi, bsdfFlags);
                            if (!f.black()) {
                                // delta lights are not weighted (integrator.cpp:57-58)
                                const float weight = light_is_delta(Ll) ? 1.f : power_heuristic(illumPdf, scatteringPdf);
#pragma unroll
                                for (int c = 0; c < NL; ++c) CL.c[c] = f.c[c] * ls.radiance * weight / illumPdf;
                                pf |= kHasCL;
                                // shadow ray (VisibilityEvaluator::unoccluded)
                                float4 so, sd;
                                if (ls.vis_kind == 1) {
                                    const v3 dd = sub(ls.target, hr.p);
                                    const v3 oo = spawn_origin(hr.p, hr.n, dd);
                                    so = make_float4(oo.x, oo.y, oo.z, kShadowEpsilon);
                                    sd = make_float4(dd.x, dd.y, dd.z, 1.f - kShadowEpsilon);
                                } else {
                                    const v3 oo = spawn_origin(hr.p, hr.n, wi);
                                    so = make_float4(oo.x, oo.y, oo.z, kShadowEpsilon);
                                    sd = make_float4(wi.x, wi.y, wi.z, __int_as_float(0x7f800000));
                                }
                                const uint32_t pos = coalesced_append(&A.cnt->n_shadow, true);
                                if (pos < A.scap) {
                                    A.sray_o[pos] = so;
                                    A.sray_d[pos] = sd;
                                    A.stag[pos] = shadow_tag(slot, (uint32_t)li, 0u);
                                } else {
                                    atomicAdd(&A.cnt->err, 1);
                                }
                            }
                        }
                        // BSDF sampling term (none for delta lights, integrator.cpp:66)
                        if (!light_is_delta(Ll)) {
                            Spec<NL> f;
                            int sampledType = 0;
                            bsdf_sample<STD>(b, hr.wo, wi, usx, usy, scatteringPdf, bsdfFlags, sampledType, f);
                            const float ad = absdot(wi, b.ns);
#pragma unroll
                            for (int c = 0; c < NL; ++c) f.c[c] *= ad;
                            const bool sampledSpecular = (sampledType & kBsdfSpecular) != 0;
                            if (!f.black() && scatteringPdf > 0) {
                                float weight = 1.f;
                                bool ok = true;
                                if (!sampledSpecular) {
                                    illumPdf = light_pdf_li(Ll, J.soup, hr, wi);
                                    if (illumPdf == 0) ok = false;
                                    else weight = power_heuristic(scatteringPdf, illumPdf);
                                }
                                const float Lrad = Ll.radiance;  // le() of the hit light, or of the environment on a miss
                                if (ok && Lrad != 0.f) {
#pragma unroll
                                    for (int c = 0; c < NL; ++c)
                                        CS.c[c] = f.c[c] * Lrad * 1.f * weight / scatteringPdf;
                                    pf |= kHasCS;
                                    const v3 oo = spawn_origin(hr.p, hr.n, wi);
                                    const uint32_t pos = coalesced_append(&A.cnt->n_shadow, true);
                                    if (pos < A.scap) {
                                        A.sray_o[pos] = make_float4(oo.x, oo.y, oo.z, kShadowEpsilon);
                                        A.sray_d[pos] = make_float4(wi.x, wi.y, wi.z, __int_as_float(0x7f800000));
                                        A.stag[pos] = shadow_tag(slot, (uint32_t)li, 1u);
                                    } else {
                                        atomicAdd(&A.cnt->err, 1);
                                    }
                                }
                            }
                        }
                        A.pflags[(size_t)li * A.cap + slot] = pf;
                        if (pf & kHasCL) store_spec<NL>(A.CL + (size_t)li * NL * A.cap, A.cap, slot, CL);
                        if (pf & kHasCS) store_spec<NL>(A.CS + (size_t)li * NL * A.cap, A.cap, slot, CS);
                    }
                    A.head[slot].rng = rng.state;
                }
            }
        }
        const uint32_t pos = warp_append(STD ? &A.cnt->n_cont_std : &A.cnt->n_cont, alive);
        if (alive) A.q_cont[STD ? A.cap - 1 - pos : pos] = slot;
    }
    warp_count(&A.cnt->bounces, shaded);
}

struct NeeRayItem {
    const RenderArgs *A;
    const JobDev *J;
    const WideNode *nodes;
    uint32_t n_nodes;
    const float4 *tris;
    uint32_t n_tris;
    uint32_t q, kind, slot, li;
    bool any_hit;
    RayPre ray;
    TravState st;
    __device__ void bind_job0() {  // every path in job 0: its scene once, not per ray
        J = A->job0;
        nodes = J->nodes;
        n_nodes = J->n_nodes;
        tris = J->tris;
        n_tris = J->n_tri;
    }
    __device__ bool begin(uint32_t qq) {
        q = qq;
        const uint32_t tag = A->stag[q];
        kind = tag & 1u;
        li = (tag >> 1) & 63u;
        slot = tag >> 7;
        if (!A->job0) {
            J = &A->jobs[A->head[slot].job];
            nodes = J->nodes;
            n_nodes = J->n_nodes;
            tris = J->tris;
            n_tris = J->n_tri;
        }
        ray = ray_precompute(A->sray_o[q], A->sray_d[q]);
        // shadow rays stop at the first hit when no triangle emits; a MIS ray towards the
        // environment only asks whether it escapes, so any triangle hit ends it as well
        any_hit = kind == 0 ? J->any_hit_ok != 0 : J->lights[li].type == FL_LIGHT_ENV;
        trav_init(st, ray);
        return true;
    }
    __device__ void finish() {
        const uint32_t sl = li * A->cap + slot;
        TraceResult res = st.res;
        uint32_t bit = 0;
        if (kind == 0) {
            // VisibilityEvaluator::unoccluded: no hit, or the closest hit is emissive
            const bool unocc = res.id < 0 || J->tri_light[res.id] >= 0;
            bit = unocc ? kVisOK : 0u;
        } else {
            add_spheres(*J, ray, res);
            const LightDev Ll = J->lights[li];
            bool ok = false;
            if (res.id == -1) ok = Ll.type == FL_LIGHT_ENV;
            else if (prim_light(*J, res.id) == (int)li) {
                const int4 h = make_int4(res.id, __float_as_int(res.t), 0, 0);
                const Hit hr = make_hit(*J, A->sray_o[q], A->sray_d[q], h);
                ok = dot(hr.n, mk(-ray.dx, -ray.dy, -ray.dz)) > 0.f;
            }
            bit = ok ? kMisOK : 0u;
        }
        if (bit) atomicOr(&A->pflags[sl], bit);
    }
};

// shadow rays (kind 0) and MIS rays (kind 1), persistent
template <bool COUNT>
__global__ void __launch_bounds__(128, kRenderRays2Blocks) k_trace_rays2(RenderArgs A) {
    const uint32_t n = min(load_count(&A.cnt->n_shadow), A.scap);
    bool err = false;
    TraceStats st;
    NeeRayItem it;
    it.A = &A;
    if (A.job0) it.bind_job0();
    __shared__ uint2 stack[trav_stack_smem_bytes(128) / sizeof(uint2)];
    __shared__ uint4 top[kSmemNodeWords];
    const uint32_t n_top = trav_stage_top(top, A.job0 ? it.nodes : nullptr, A.job0 ? it.n_nodes : 0u);
    persistent_trace<kRenderTraceSteps, COUNT>(it, &A.cnt->fetch_rays2, n, err, st, stack, top, n_top);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&A.cnt->shadow_rays, (unsigned long long)n);
        atomicAdd(&A.cnt->rays, (unsigned long long)n);
    }
    if (COUNT) {
        warp_count(&A.cnt->nodes, st.nodes);
        warp_count(&A.cnt->tris, st.tris);
    }
    if (err) atomicAdd(&A.cnt->err, 1);
}

// A training record at a Lambert vertex (the path's first two): the record is closed by
// finish_path with the radiance the path gathers after it.
template <int NL>
__device__ inline void guide_record(const RenderArgs &A, uint32_t slot, const Hit &hr, float lambda0, v3 wi,
                                    float pdf, const Spec<NL> &beta_after, const Spec<NL> &L_before) {
    int r = -1;
    if (A.g.rec_idx[slot] == kNoRecord) r = 0;
    else if (A.g.rec_idx[(size_t)A.cap + slot] == kNoRecord) r = 1;
    if (r < 0) return;
    const uint32_t pos = atomicAdd(A.g.rec_count, 1u);
    if (pos >= A.g.rec_cap) return;
    const v3 nf = dot(hr.n, hr.wo) < 0.f ? neg(hr.n) : hr.n;
    float *R = A.g.rec + (size_t)pos * kRecFloats;
    float4 *R4 = reinterpret_cast<float4 *>(R);
    R4[0] = make_float4(hr.p.x, hr.p.y, hr.p.z, nf.x);
    R4[1] = make_float4(nf.y, nf.z, lambda0, wi.x);
    R4[2] = make_float4(wi.y, wi.z, pdf, 0.f);
    R4[3] = make_float4(beta_after.c[0], beta_after.c[1], beta_after.c[2], beta_after.c[3]);
    R4[4] = make_float4(L_before.c[0], L_before.c[1], L_before.c[2], L_before.c[3]);
    A.g.rec_idx[(size_t)r * A.cap + slot] = pos;
}

// Guide inference for the paths that hit a Lambert surface this bounce: 16 points per warp
// on the tensor cores, mixture parameters to A.g.mix. Dynamic shared memory: the weights
// plus, per warp, 16 feature rows that the 16 head rows overwrite once the first layer has
// read them (16 x 88 halves = 16 x 44 floats; guide_infer_smem_bytes).
constexpr int kInferWarps = 8;
static_assert(kLdIn * 2 == kHeadLd * 4, "head rows alias the feature rows");
inline size_t guide_infer_smem_bytes() { return (size_t)kSmWHalves * 2 + (size_t)kInferWarps * 16 * kLdIn * 2; }
template <int NL>
__global__ void __launch_bounds__(32 * kInferWarps, 3) k_guide_infer(RenderArgs A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    __half *sw = reinterpret_cast<__half *>(gsm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __half *X = reinterpret_cast<__half *>(gsm + kSmWHalves * 2) + warp * 16 * kLdIn;
    float *head = reinterpret_cast<float *>(X);
    const int cls = 1 + FL_MAT_LAMBERT;
    const uint32_t n = load_count(&A.cnt->n_class[cls]);
    if ((uint32_t)blockIdx.x * kInferWarps * 16 >= n) return;
    guide_stage_weights(sw, A.g.w);
    const uint32_t *q = A.q_class + (size_t)cls * A.cap;
    for (uint32_t chunk = blockIdx.x * kInferWarps + warp; chunk * 16 < n; chunk += gridDim.x * kInferWarps) {
        const uint32_t i = chunk * 16 + (lane & 15);
        const bool valid = i < n;
        uint32_t slot = 0;
        __half *row = X + (lane & 15) * kLdIn;
        if (valid) {
            slot = q[i];
            const JobDev &J = A.jobs[A.head[slot].job];
            const Hit hr = make_hit(J, A.ray_o[slot], A.ray_d[slot], A.hit[slot]);
            const v3 nf = dot(hr.n, hr.wo) < 0.f ? neg(hr.n) : hr.n;
            float pn[3];
            guide_normalise(A.g.bmin, A.g.binv, hr.p, pn);
            const float nn[3] = {nf.x, nf.y, nf.z};
            guide_encode_part(pn, nn, (A.head[slot].lambda0 - 380.f) * (1.f / 340.f), lane >> 4, row);
        } else {
            uint4 *d = reinterpret_cast<uint4 *>(row + 40 * (lane >> 4));
#pragma unroll
            for (int k = 0; k < 5; ++k) d[k] = make_uint4(0, 0, 0, 0);
        }
        __syncwarp();
        guide_forward_warp(sw, X, nullptr, 0, head);
        __syncwarp();
        if (valid && lane < 16) guide_mixture(head + lane * kHeadLd, A.g.mix + (size_t)slot * kMixFloats, true);
        __syncwarp();
    }
}

template <int NL, bool GUIDE = false, bool STD = false>
__global__ void FL_CONT_BOUNDS k_continue(RenderArgs A) {
    __shared__ SmemTables sm;
    stage_tables(sm, A.tab, NL != 60);
    const uint32_t n = load_count(STD ? &A.cnt->n_cont_std : &A.cnt->n_cont);
    FL_WARP_UNIFORM_LOOP(q, n) {
        const bool active = q < n;
        bool alive = false;
        uint32_t slot = 0;
        if (active) {
            slot = A.q_cont[STD ? A.cap - 1 - q : q];
            const JobDev &J = A.jobs[A.head[slot].job];
            const int4 h = A.hit[slot];
            const uint32_t fl = A.head[slot].flags;
            const uint32_t bounce = fl & 0xffu;
            const float4 o4 = A.ray_o[slot], d4 = A.ray_d[slot];
            const Hit hr = make_hit(J, o4, d4, h);
            const float lambda0 = A.head[slot].lambda0;
            Bsdf<NL> b;
            make_bsdf<NL, STD>(J, A.tab, sm, hr, lambda0, b);
            Spec<NL> beta, L;
            load_spec<NL>(A.beta, A.cap, slot, beta);
            load_spec<NL>(A.L, A.cap, slot, L);
            if (bsdf_num_components<STD>(b, kBsdfAll & ~kBsdfSpecular) > 0) {
                // uniform_sample_all_lights: sum of the per-light estimate_direct results
                Spec<NL> Ls;
                Ls.set(0.f);
                for (int li = 0; li < J.n_lights; ++li) {
                    const uint32_t pf = A.pflags[(size_t)li * A.cap + slot];
                    Spec<NL> Ld;
                    Ld.set(0.f);
                    if ((pf & kHasCL) && (pf & kVisOK)) {
                        Spec<NL> c;
                        load_spec<NL>(A.CL + (size_t)li * NL * A.cap, A.cap, slot, c);
#pragma unroll
                        for (int k = 0; k < NL; ++k) Ld.c[k] += c.c[k];
                    }
                    if ((pf & kHasCS) && (pf & kMisOK)) {
                        Spec<NL> c;
                        load_spec<NL>(A.CS + (size_t)li * NL * A.cap, A.cap, slot, c);
#pragma unroll
                        for (int k = 0; k < NL; ++k) Ld.c[k] += c.c[k];
                    }
#pragma unroll
                    for (int k = 0; k < NL; ++k) Ls.c[k] += Ld.c[k];
                }
#pragma unroll
                for (int k = 0; k < NL; ++k) L.c[k] += beta.c[k] * Ls.c[k];
            }
            // continuation (pathintegrator.cpp:46-84)
            Pcg32 rng;
            rng.state = A.head[slot].rng;
            rng.inc = 3u;
            const v3 wo = mk(-d4.x, -d4.y, -d4.z);
            v3 wi = mk(0.f, 0.f, 0.f);
            float pdf = 0.f;
            int sflags = 0;
            Spec<NL> f;
            // guiding at Lambert vertices: one-sample MIS between the learned mixture
            // (probability c) and the BSDF; an extra number picks the technique and the lobe
            const float *gm = nullptr;
            float c_sel = 0.f, u_sel = 1.f;
            if constexpr (GUIDE) {
                if (!STD && b.type == FL_MAT_LAMBERT && A.g.select > 0.f && lambert_count(fl) < kGuidedVertices) {
                    gm = A.g.mix + (size_t)slot * kMixFloats;
                    if (gm[0] >= 0.f) {
                        c_sel = A.g.learned_select ? gm[kMixSelect] : A.g.select;
                        u_sel = rng.nextf();
                    }
                }
            }
            const float ux = rng.nextf(), uy = rng.nextf();
            if (GUIDE && u_sel < c_sel) {
                wi = guide_mixture_sample(gm, u_sel / c_sel, ux, uy);
                bsdf_eval<STD>(b, wo, wi, kBsdfAll, f);
                pdf = bsdf_pdf<STD>(b, wo, wi, kBsdfAll);
                sflags = kBsdfDiffuse | kBsdfReflection;
            } else {
                bsdf_sample<STD>(b, wo, wi, ux, uy, pdf, kBsdfAll, sflags, f);
            }
            if (GUIDE && c_sel > 0.f && !(f.black() || pdf == 0))
                pdf = c_sel * guide_mixture_pdf(gm, wi) + (1.f - c_sel) * pdf;
            bool stop = f.black() || pdf == 0;
            // the depth of the sampled lobe's kind ends the path at exactly that bounce
            // (pathintegrator.cpp:55-65)
            const int bi = (int)bounce;
            if (!stop && J.depth[0] == bi && (sflags & kBsdfDiffuse)) stop = true;
            if (!stop && ((J.depth[1] == bi && (sflags & kBsdfSpecular)) || (J.depth[1] == bi && (sflags & kBsdfGlossy))))
                stop = true;
            if (!stop && J.depth[2] == bi && (sflags & kBsdfTransmission)) stop = true;
            if (!stop) {
                const float ad = absdot(wi, b.ns);
#pragma unroll
                for (int k = 0; k < NL; ++k) beta.c[k] *= f.c[k] * ad / pdf;
                if constexpr (GUIDE && NL == 4) {
                    if (!STD && A.g.record && b.type == FL_MAT_LAMBERT)
                        guide_record(A, slot, hr, lambda0, wi, pdf, beta, L);
                }
                const bool spec_b = (sflags & kBsdfSpecular) != 0;
                float etaScale = A.head[slot].eta_scale;
                if ((sflags & kBsdfSpecular) && (sflags & kBsdfTransmission)) {
                    const float eta = b.eta;
                    etaScale *= (dot(wo, hr.n) > 0) ? (eta * eta) : 1.f / (eta * eta);
                }
                const v3 no = spawn_origin(hr.p, hr.n, wi);
                float mx = beta.c[0] * etaScale;
#pragma unroll
                for (int k = 1; k < NL; ++k) mx = fmaxf(mx, beta.c[k] * etaScale);
                if (mx < J.rr_threshold && bi > 3) {
                    float qq = 1.f - mx;
                    if (qq < 0.05f) qq = 0.05f;
                    if (rng.nextf() < qq) stop = true;
                    else {
#pragma unroll
                        for (int k = 0; k < NL; ++k) beta.c[k] /= 1.f - qq;
                    }
                }
                if (!stop && bi + 1 >= J.bounce_cap) {
                    // unequal lobe depths: a path still going at the bounce bound is cut
                    stop = true;
                    atomicAdd(&A.cnt->cut, 1u);
                }
                if (!stop) {
                    alive = true;
                    store_spec<NL>(A.beta, A.cap, slot, beta);
                    A.head[slot].eta_scale = etaScale;
                    uint32_t nfl = (bounce + 1u) | (spec_b ? 0x100u : 0u);
                    if constexpr (GUIDE) {
                        const uint32_t lc = lambert_count(fl) + (!STD && b.type == FL_MAT_LAMBERT ? 1u : 0u);
                        nfl |= (lc < 3u ? lc : 3u) << 9;
                    }
                    A.head[slot].flags = nfl;
                    A.ray_o[slot] = make_float4(no.x, no.y, no.z, kShadowEpsilon);
                    A.ray_d[slot] = make_float4(wi.x, wi.y, wi.z, __int_as_float(0x7f800000));
                }
            }
            A.head[slot].rng = rng.state;
            if (alive) store_spec<NL>(A.L, A.cap, slot, L);
            else finish_path<NL>(A, J, sm, slot, L);
        }
        const uint32_t pos = warp_append(&A.cnt->n_next, alive);
        if (alive) A.q_next[pos] = slot;
    }
}

static __global__ void k_resolve(const double *__restrict__ film, uint32_t n_pix, double inv_spp, float *__restrict__ rgb) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_pix; p += gridDim.x * blockDim.x) {
        const float x = (float)(film[3 * (size_t)p] * inv_spp);
        const float y = (float)(film[3 * (size_t)p + 1] * inv_spp);
        const float z = (float)(film[3 * (size_t)p + 2] * inv_spp);
        // xyz_to_rgb, color/spectrumoperations.cpp:58-66
        rgb[3 * (size_t)p + 0] = 3.240479f * x - 1.537150f * y - 0.498535f * z;
        rgb[3 * (size_t)p + 1] = -0.969256f * x + 1.875991f * y + 0.041556f * z;
        rgb[3 * (size_t)p + 2] = 0.055648f * x - 0.204043f * y + 1.057311f * z;
    }
}

// ------------------------------------------------------------------------------ host side

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// Iterations per graph replay of a streaming wave, and the most paths one descriptor lists.
constexpr int kStreamIters = 8;
static_assert(kStreamIters % 2 == 0, "a replay starts at queue parity 0");
constexpr unsigned long long kStreamDescPaths = 1ull << 31;
// Default path slots of a streaming wave. More slots give each iteration's kernels more
// rays to share the GPU: the 1,048,578-triangle procedural frame (1920x1080, 64 spp, depth
// 16) measured 1,430 Mrays/s with 2^20 slots, 1,582 with 2^21, 1,668 with 2^22 and 1,685
// with 2^23 (3.3 GB of state with two lights). The 60-bin mode has 15x the spectra per slot.
constexpr size_t kWavePathsHero = (size_t)1 << 23;
constexpr size_t kWavePathsBins60 = (size_t)1 << 21;
// The wave state of a render lives in the context scratch, at most this many bytes.
constexpr size_t kWaveScratchBytes = (size_t)16 << 30;
// bytes of wave state per path slot
inline size_t wave_bytes_per_slot(int NL, int nl) {
    return 101 + 4 * kShadeClasses + 8 * (size_t)NL + 8 * (size_t)NL * nl + 4 * (size_t)nl + 72 * (size_t)nl;
}

// The device buffers of a wavefront: job table, wave descriptor, path state and queues.
struct WaveBuffers {
    RenderArgs A;
    uint32_t *qa, *qb;
    // streaming waves set A.slot_free / free_count / free_off to these
    uint8_t *slot_free;
    uint32_t *free_count, *free_off;
    JobDev *d_jobs;
    WaveDesc *d_wave;
    size_t cap;
};

// Lays the buffers out in `fixed` (fixed_bytes) or in the context scratch. The wave holds
// at most cap_request paths and no more than the buffer allows.
inline fl_status wave_buffers(Context *ctx, int NL, int nl, size_t cap_request, void *fixed, size_t fixed_bytes,
                              WaveBuffers &W) {
    const size_t per_slot = wave_bytes_per_slot(NL, nl);
    const size_t head = align_up(sizeof(WaveCounters)) + align_up(sizeof(JobDev) * kMaxJobs) + align_up(sizeof(WaveDesc));
    const size_t budget = fixed ? fixed_bytes : kWaveScratchBytes;
    if (budget < head + 32 * 256 + 128 * per_slot) {
        set_error(ctx, "render state does not fit the fixed scratch buffer");
        return FL_ERR_CAPACITY;
    }
    size_t cap = std::min(cap_request, (budget - head - 32 * 256) / per_slot);
    cap = std::max<size_t>(128, cap & ~(size_t)127);
    if (cap >= kMaxWaveSlots || cap * (size_t)std::max(nl, 1) >= ((size_t)1 << 31) || nl > 64) {
        set_error(ctx, "wave too large for the shadow-ray tags");
        return FL_ERR_INVALID;
    }
    const size_t scap = cap * 2 * (size_t)nl;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes ? bytes : 1); return o; };
    const size_t o_cnt = take(sizeof(WaveCounters)), o_jobs = take(sizeof(JobDev) * kMaxJobs),
                 o_wave = take(sizeof(WaveDesc));
    const size_t o_head = take(sizeof(PathHead) * cap), o_beta = take(4 * NL * cap), o_L = take(4 * NL * cap);
    const size_t o_ro = take(16 * cap), o_rd = take(16 * cap), o_hit = take(16 * cap);
    const size_t o_CL = take(4 * (size_t)NL * nl * cap), o_CS = take(4 * (size_t)NL * nl * cap);
    const size_t o_pf = take(4 * (size_t)nl * cap);
    const size_t o_so = take(16 * scap), o_sd = take(16 * scap), o_st = take(4 * scap);
    const size_t o_qa = take(4 * cap), o_qb = take(4 * cap), o_qc = take(4 * cap);
    const size_t o_qk = take(4 * cap * kShadeClasses);
    const size_t o_free = take(cap), o_fc = take(4 * (size_t)free_chunks(cap)), o_fo = take(4 * (size_t)free_chunks(cap));
    void *base = fixed;
    if (!fixed) {
        fl_status rc = ensure_scratch(ctx, off, &base);
        if (rc) return rc;
    } else if (off > fixed_bytes) {
        set_error(ctx, "render state does not fit the fixed scratch buffer");
        return FL_ERR_CAPACITY;
    }
    char *B = static_cast<char *>(base);
    RenderArgs &A = W.A;
    A = RenderArgs{};
    const SpectralTablesDev &T = ctx->tables;
    A.tab = TablesArg{T.cie_lambda0, T.n_cie, T.cie_y_integral, T.rgb_lambda0, T.rgb_lambda1, T.n_rgb,
                      T.cie_xyz, T.rgb_bases, T.binned};
    W.d_jobs = reinterpret_cast<JobDev *>(B + o_jobs);
    W.d_wave = reinterpret_cast<WaveDesc *>(B + o_wave);
    A.jobs = W.d_jobs;
    A.wave = W.d_wave;
    A.nl = nl;
    A.cap = (uint32_t)cap;
    A.scap = (uint32_t)scap;
    A.cnt = reinterpret_cast<WaveCounters *>(B + o_cnt);
    A.head = reinterpret_cast<PathHead *>(B + o_head);
    A.beta = reinterpret_cast<float *>(B + o_beta);
    A.L = reinterpret_cast<float *>(B + o_L);
    A.ray_o = reinterpret_cast<float4 *>(B + o_ro);
    A.ray_d = reinterpret_cast<float4 *>(B + o_rd);
    A.hit = reinterpret_cast<int4 *>(B + o_hit);
    A.CL = reinterpret_cast<float *>(B + o_CL);
    A.CS = reinterpret_cast<float *>(B + o_CS);
    A.pflags = reinterpret_cast<uint32_t *>(B + o_pf);
    A.sray_o = reinterpret_cast<float4 *>(B + o_so);
    A.sray_d = reinterpret_cast<float4 *>(B + o_sd);
    A.stag = reinterpret_cast<uint32_t *>(B + o_st);
    A.q_cont = reinterpret_cast<uint32_t *>(B + o_qc);
    A.q_class = reinterpret_cast<uint32_t *>(B + o_qk);
    W.slot_free = reinterpret_cast<uint8_t *>(B + o_free);
    W.free_count = reinterpret_cast<uint32_t *>(B + o_fc);
    W.free_off = reinterpret_cast<uint32_t *>(B + o_fo);
    W.qa = reinterpret_cast<uint32_t *>(B + o_qa);
    W.qb = reinterpret_cast<uint32_t *>(B + o_qb);
    W.cap = cap;
    return FL_OK;
}

// Blocks per SM of the grid-stride shading kernels: as many as are resident at once, so
// that every block of a launch runs from the start (a grid of more blocks than fit leaves a
// second, partial wave of blocks that starts late and ends the launch alone).
// FL_SHADE_GRID_OCC 0: 8 per SM whatever fits.
#ifndef FL_SHADE_GRID_OCC
#define FL_SHADE_GRID_OCC 1
#endif
struct ShadeShapes {
    int shade, shade_std, cont, cont_std;
};
template <class K>
inline int resident_blocks(K kernel) {
    int b = 0;
    if (!FL_SHADE_GRID_OCC || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 128, 0) != cudaSuccess || b <= 0) {
        cudaGetLastError();
        b = 8;
    }
    return b;
}
// computed on first use; call it before a stream capture of the bounces
template <int NL, bool GUIDE>
const ShadeShapes &shade_shapes() {
    static const ShadeShapes s{resident_blocks(k_shade<NL>), resident_blocks(k_shade<NL, true>),
                               resident_blocks(k_continue<NL, GUIDE>), resident_blocks(k_continue<NL, GUIDE, true>)};
    return s;
}

// Enqueues bounces [b_begin, b_end) of a wave on `st`. Bounce b reads the trace queue of
// parity b (qa for even b) and appends survivors to the other one. With `stream` each is an
// iteration of a streaming wave: it first starts new paths in the free slots (k_free_count,
// k_stream_step, k_regen). Launch shapes do not depend on the wave's content (kernels read
// their counts from device memory).
template <int NL, bool GUIDE = false>
void enqueue_bounces(const WaveBuffers &W, int b_begin, int b_end, bool count, RenderProfile *prof, int sms,
                     cudaStream_t st, bool standard, bool stream = false) {
    RenderArgs A = W.A;
    const ShadeShapes &sh = shade_shapes<NL, GUIDE>();
    const int g_trace = sms * 16;
    for (int b = b_begin; b < b_end; ++b) {
        A.q_trace = (b & 1) ? W.qb : W.qa;
        A.q_next = (b & 1) ? W.qa : W.qb;
        if (stream) {
            // streaming: survivors plus new paths in the lowest free slots
            const uint32_t nc = free_chunks(A.cap);
            k_free_count<<<nc, 256, 0, st>>>(A);
            k_stream_step<<<1, 1024, 0, st>>>(A);
            k_regen<NL><<<nc, 256, 0, st>>>(A);
            prof->launches += 3;
        } else if (b > 0) {
            k_advance<<<1, 1, 0, st>>>(A.cnt);
            prof->launches += 1;
        }
        prof->mark(0, st);
        if (count) k_trace_paths<true><<<g_trace, 128, 0, st>>>(A);
        else k_trace_paths<false><<<g_trace, 128, 0, st>>>(A);
        prof->mark(0, st);
        prof->mark(1, st);
        k_shade<NL><<<sms * sh.shade, 128, 0, st>>>(A);
        if (standard) k_shade<NL, true><<<sms * sh.shade_std, 128, 0, st>>>(A);
        prof->mark(1, st);
        prof->mark(2, st);
        if (count) k_trace_rays2<true><<<g_trace, 128, 0, st>>>(A);
        else k_trace_rays2<false><<<g_trace, 128, 0, st>>>(A);
        prof->mark(2, st);
        prof->mark(3, st);
        if constexpr (GUIDE) {
            if (A.g.select > 0.f) {
                k_guide_infer<NL><<<sms * 3, 32 * kInferWarps, guide_infer_smem_bytes(), st>>>(A);
                prof->launches += 1;
            }
        }
        k_continue<NL, GUIDE><<<sms * sh.cont, 128, 0, st>>>(A);
        if (standard) k_continue<NL, GUIDE, true><<<sms * sh.cont_std, 128, 0, st>>>(A);
        prof->mark(3, st);
        prof->launches += standard ? 6 : 4;
    }
}

// Enqueues one wave: camera rays of the samples in *W.d_wave, then bounces 0..depth. The
// sequence can be captured once into a CUDA graph and replayed for every wave.
// `standard`: the wave may hold StandardSurface materials, shaded by their own kernel instances.
template <int NL, bool GUIDE = false>
void enqueue_wave(const WaveBuffers &W, int depth, bool count, RenderProfile *prof, int sms, cudaStream_t st,
                  bool standard) {
    RenderArgs A = W.A;
    A.q_trace = W.qa;
    A.q_next = W.qb;
    k_raygen<NL><<<std::min<uint32_t>(((uint32_t)W.cap + 127) / 128, (uint32_t)sms * 32), 128, 0, st>>>(A);
    prof->launches += 1;
    enqueue_bounces<NL, GUIDE>(W, 0, depth + 1, count, prof, sms, st, standard);
}

// With unequal lobe depths a path is ended only by the depth of the lobe kind it samples,
// at that exact bounce, so it can outlive the deepest depth. After a wave's fixed bounces
// 0..first_bounce - 1 the paths still alive run further bounces, kTailBounces per check of
// the live count, until none is left; k_continue cuts what reaches FL_MAX_BOUNCES.
constexpr int kTailBounces = 4;
template <int NL, bool GUIDE = false>
fl_status run_tail(Context *ctx, const WaveBuffers &W, int first_bounce, bool count, RenderProfile *prof, int sms,
                   cudaStream_t st, bool standard) {
    for (int b = first_bounce; b < FL_MAX_BOUNCES; b += kTailBounces) {
        uint32_t live = 0;
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(&live, &W.A.cnt->n_next, sizeof(live), cudaMemcpyDeviceToHost, st));
        FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        if (live == 0) break;
        enqueue_bounces<NL, GUIDE>(W, b, std::min(b + kTailBounces, FL_MAX_BOUNCES), count, prof, sms, st, standard);
        FL_CUDA_TRY(ctx, cudaGetLastError());
    }
    return FL_OK;
}

// FL_ERR_TRAVERSAL when a traversal, queue or bounce bound was hit during a render (the
// image holds everything else), with the counts in the context's message.
inline fl_status render_bounds_status(Context *ctx, const WaveCounters &hc) {
    if (!hc.err && !hc.cut) return FL_OK;
    std::string m;
    if (hc.err) m = std::to_string(hc.err) + " traversal or queue bound hits during the render";
    if (hc.cut) m += (m.empty() ? "" : "; ") + std::to_string(hc.cut) + " paths still alive at FL_MAX_BOUNCES were cut";
    set_error(ctx, m);
    return FL_ERR_TRAVERSAL;
}

// The job record of one scene + camera + parameters (fl_render's single job).
inline JobDev job_of(const Scene *s, const CamDev &cam, const fl_render_params &p, double *d_film) {
    JobDev j{};
    j.nodes = s->nodes;
    j.n_nodes = s->n_nodes;
    j.tris = s->tris;
    j.n_tri = s->n_tri;
    j.soup = s->soup;
    j.tri_material = s->tri_material;
    j.tri_light = s->tri_light;
    j.materials = s->materials;
    j.mat_refl60 = s->mat_refl60;
    j.standard = s->standard;
    j.std_refl60 = s->std_refl60;
    j.uvs = s->uvs;
    j.pixels = s->pixels;
    j.images = s->images;
    j.lights = s->lights;
    j.n_lights = (int)s->n_lights;
    j.any_hit_ok = s->n_emissive_tris == 0 ? 1 : 0;
    j.has_env = s->has_env;
    j.env_radiance = s->env_radiance;
    j.has_spheres = 0;
    for (const auto &l : s->lights_host) j.has_spheres |= (l.type == FL_LIGHT_SPHERE) ? 1 : 0;
    j.cam = cam;
    j.spp = p.spp;
    lobe_depths(p, j.depth);
    // equal depths end every path by bounce depth (no cut); unequal ones run to the bound
    j.bounce_cap = depths_equal(p) ? j.depth[0] + 1 : FL_MAX_BOUNCES;
    j.rr_threshold = p.rr_threshold;
    j.sample_offset = p.sample_offset;
    j.n_pix = (uint32_t)((uint64_t)cam.W * (uint64_t)cam.H);
    j.film = d_film;
    j.corrected_ggx = (p.flags & FL_RENDER_CORRECTED_GGX) ? 1 : 0;
    return j;
}

// Renders all samples of one image into d_film (FP64 XYZ sums) wave by wave, without host
// synchronisation. Instantiated per spectral mode in its own translation unit (the 60-bin
// one without FMA contraction).
template <int NL>
fl_status render_waves(Scene *s, const CamDev &cam, const fl_render_params &p, double *d_film,
                       WaveCounters *h_cnt, RenderProfile *prof, cudaStream_t st, void *fixed_scratch = nullptr,
                       size_t fixed_bytes = 0, const LiRays *li = nullptr) {
    Context *ctx = s->ctx;
    const unsigned long long n_pix = (unsigned long long)cam.W * (unsigned long long)cam.H;
    const unsigned long long total = n_pix * (unsigned long long)p.spp;
    size_t cap_req = p.wave_paths > 0 ? (size_t)p.wave_paths : (NL == 60 ? kWavePathsBins60 : kWavePathsHero);
    cap_req = std::min<size_t>(cap_req, (size_t)total);
    WaveBuffers W;
    fl_status rc = wave_buffers(ctx, NL, (int)s->n_lights, cap_req, fixed_scratch, fixed_bytes, W);
    if (rc) return rc;
    JobDev j = job_of(s, cam, p, d_film);
    if (li) j.li = *li;
    W.A.job0 = W.d_jobs;  // one job: every path's scene is job 0's
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(W.d_jobs, &j, sizeof(JobDev), cudaMemcpyHostToDevice, st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(W.A.cnt, 0, sizeof(WaveCounters), st));
    const bool count = (p.flags & FL_RENDER_COUNT) != 0;
    const bool standard = s->ext_kernels;
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const size_t desc_bytes = offsetof(WaveDesc, seg) + sizeof(WaveSeg);
    const int bounce_cap = j.bounce_cap;
    // Streaming waves: slots of ended paths take the descriptor's next paths every
    // iteration, so the wave stays full until its paths run out and the late bounces of a
    // few long paths are paid once per descriptor, not once per wave of cap paths. The
    // host looks at the counters after every kStreamIters iterations (one graph replay).
    W.A.slot_free = W.slot_free;
    W.A.free_count = W.free_count;
    W.A.free_off = W.free_off;
    // Replay one captured graph per kStreamIters iterations. Not used by the allocation-free
    // path (instantiating a graph allocates), when every launch is timed with events, nor by
    // fl_li (its small batches would replace the render's graph with one of their own size).
    const bool use_graph = !fixed_scratch && !prof->on && !li;
    shade_shapes<NL, false>();  // launch shapes, outside any capture
    if (use_graph && (!ctx->wave_graph || ctx->graph_base != W.A.cnt || ctx->graph_cap != W.cap ||
                      ctx->graph_depth != kStreamIters || ctx->graph_nl_mode != NL || ctx->graph_count != (int)count ||
                      ctx->graph_std != (int)standard)) {
        if (ctx->wave_graph) {
            cudaGraphExecDestroy(ctx->wave_graph);
            ctx->wave_graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        RenderProfile off;
        FL_CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_bounces<NL>(W, 0, kStreamIters, count, &off, sms, st, standard, true);
        FL_CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
        cudaError_t e = cudaGraphInstantiate(&ctx->wave_graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            ctx->wave_graph = nullptr;
            return cuda_status(ctx, e, "wave graph instantiation");
        }
        ctx->graph_base = W.A.cnt;
        ctx->graph_cap = W.cap;
        ctx->graph_depth = kStreamIters;
        ctx->graph_nl_mode = NL;
        ctx->graph_count = (int)count;
        ctx->graph_std = (int)standard;
    }
    const uint32_t per_iter = standard ? 9u : 7u;  // launches per iteration
    for (unsigned long long wb = 0; wb < total; wb += kStreamDescPaths) {
        WaveDesc d;
        d.n_wave = (uint32_t)std::min<unsigned long long>(kStreamDescPaths, total - wb);
        d.n_seg = 1;
        d.seg[0] = WaveSeg{0u, 0u, d.n_wave, 0u, wb, 0ull};
        // pageable source: the copy is staged before the call returns, so `d` may be reused
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(W.d_wave, &d, desc_bytes, cudaMemcpyHostToDevice, st));
        k_stream_init<<<std::min<uint32_t>(((uint32_t)W.cap + 127) / 128, (uint32_t)sms * 8), 128, 0, st>>>(W.A);
        prof->launches += 1;
        // every path ends within bounce_cap bounces, so each run of bounce_cap + 1 iterations
        // frees every slot that was busy at its start
        const unsigned long long max_iters =
            ((unsigned long long)d.n_wave / W.cap + 2ull) * (unsigned long long)(bounce_cap + 2);
        for (unsigned long long it = 0;; it += kStreamIters) {
            if (it > max_iters) {
                set_error(ctx, "streaming wave did not drain within its iteration bound");
                return FL_ERR_TRAVERSAL;
            }
            if (use_graph) {
                FL_CUDA_TRY(ctx, cudaGraphLaunch(ctx->wave_graph, st));
                prof->launches += per_iter * kStreamIters;
            } else {
                enqueue_bounces<NL>(W, 0, kStreamIters, count, prof, sms, st, standard, true);
            }
            FL_CUDA_TRY(ctx, cudaGetLastError());
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(h_cnt, W.A.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
            FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            if (h_cnt->n_next == 0 && h_cnt->next_path >= d.n_wave) break;
        }
    }
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(h_cnt, W.A.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
    return FL_OK;
}

}  // namespace fl
