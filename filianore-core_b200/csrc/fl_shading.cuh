// Device shading: BSDFs, lights and the NEE terms of the reference's path integrator,
// per path vertex, over NL spectral samples (4 hero wavelengths or the reference's 60
// fixed bins). Semantics follow, function by function:
//   BSDF evaluate/sample/pdf    src/filianore/shading/bsdf.cpp:6-151
//   LambertBRDF                 src/filianore/shading/bxdfs/lambert.cpp:6-25
//   concentric disk / cosine    src/filianore/core/shadingcore.h:65-89
//   GGX D / Lambda / VNDF       src/filianore/shading/microfacets/ggx.cpp:12-57
//   G, pdf                      src/filianore/shading/microfacets/microfacet.cpp:6-17
//   MicrofacetReflectionBRDF    src/filianore/shading/bxdfs/microfacetreflection.cpp:13-61
//   MicrofacetTransmissionBRDF  src/filianore/shading/closures/microfacettransmission.cpp:70-239
//   FresnelSpecularBXDF         src/filianore/shading/closures/fresnelspecular.cpp:18-53
//   FresnelDielectric           src/filianore/shading/fresnel/fresneldielectric.cpp:8-38 (no state)
//   FresnelConductor            src/filianore/shading/fresnel/fresnelconductor.cpp:9-33
//   StandardSurfaceMaterial     src/filianore/shading/materials/standardsurface.cpp:72-159, with
//     OrenNayarBRDF               src/filianore/shading/bxdfs/orennayar.cpp:6-62
//     FresnelBlendedDiffuseSpec.  src/filianore/shading/closures/fresnelblendeddiffspec.cpp:18-67
//     Schlick dielectric/metallic src/filianore/shading/fresnel/schlick{dielectric,metallic}.cpp
//     EstevezSheenDistribution    src/filianore/shading/microfacets/estevez.cpp:8-42
//     ClearcoatReflectionBRDF     src/filianore/shading/bxdfs/clearcoat.cpp:6-80
//   DiffuseAreaIlluminant       src/filianore/illuminants/diffusearea.cpp:12-39
//   Shape::sample / Shape::pdf  src/filianore/shapes/shape.cpp:13-41
//   Triangle::intersect/sample  src/filianore/shapes/triangle.cpp:13-154
//   estimate_direct terms       src/filianore/integrators/integrator.cpp:25-110
// Environment and sphere lights have no reference class; they follow the same
// sample_li / pdf_li / L interface.
#pragma once

#include "fl_internal.h"

namespace fl {

// sin/cos of the path sampling code. The 60-bin parity build (FL_PARITY_MATH) evaluates
// them in double and rounds once, which gives the correctly rounded float result that
// the host C library returns for std::sin/std::cos(float); the hero build uses sinf/cosf.
#if defined(FL_PARITY_MATH)
static __device__ inline float fl_sin(float x) { return (float)sin((double)x); }
static __device__ inline float fl_cos(float x) { return (float)cos((double)x); }
#else
static __device__ inline float fl_sin(float x) { return sinf(x); }
static __device__ inline float fl_cos(float x) { return cosf(x); }
#endif
// pow/exp/log of the StandardSurface lobes, rounded once from double in the parity build
#if defined(FL_PARITY_MATH)
static __device__ inline float fl_pow(float x, float y) { return (float)pow((double)x, (double)y); }
static __device__ inline float fl_exp(float x) { return (float)exp((double)x); }
static __device__ inline float fl_log(float x) { return (float)log((double)x); }
#else
static __device__ inline float fl_pow(float x, float y) { return powf(x, y); }
static __device__ inline float fl_exp(float x) { return expf(x); }
static __device__ inline float fl_log(float x) { return logf(x); }
#endif

enum : int {
    kBsdfReflection = 1 << 0,
    kBsdfTransmission = 1 << 1,
    kBsdfDiffuse = 1 << 2,
    kBsdfGlossy = 1 << 3,
    kBsdfSpecular = 1 << 4,
    kBsdfAll = 31
};

template <int NL>
struct Spec {
    float c[NL];
    __device__ inline void set(float v) {
#pragma unroll
        for (int i = 0; i < NL; ++i) c[i] = v;
    }
    __device__ inline bool black() const {
        bool b = true;
#pragma unroll
        for (int i = 0; i < NL; ++i) b = b && (c[i] == 0.f);
        return b;
    }
};

// ---------------------------------------------------------------------------- tables
// Spectral data staged in shared memory by each shading kernel.
struct SmemTables {
    // hero: CIE x/y/z at 1 nm and the 14 RGB bases; bins: the 17 x 60 binned tables
    float cie[3 * 512];
    float bases[14 * 64];
    float binned[17 * 60];
};

struct TablesArg {
    float cie_lambda0;
    int n_cie;
    float cie_y_integral;
    float rgb_lambda0, rgb_lambda1;
    int n_rgb;
    const float *cie_xyz;
    const float *rgb_bases;
    const float *binned;
};

__device__ inline void stage_tables(SmemTables &sm, const TablesArg &t, bool hero) {
    if (hero) {
        for (int i = threadIdx.x; i < 3 * t.n_cie; i += blockDim.x) {
            const int row = i / t.n_cie, col = i - row * t.n_cie;
            sm.cie[row * 512 + col] = t.cie_xyz[i];
        }
        for (int i = threadIdx.x; i < 14 * t.n_rgb; i += blockDim.x) {
            const int row = i / t.n_rgb, col = i - row * t.n_rgb;
            sm.bases[row * 64 + col] = t.rgb_bases[i];
        }
    } else {
        for (int i = threadIdx.x; i < 17 * 60; i += blockDim.x) sm.binned[i] = t.binned[i];
    }
    __syncthreads();
}

// hero wavelengths: lambda_k = lambda0 + 85 k, wrapped into [380, 720)
__device__ inline float hero_lambda(float lambda0, int k) {
    float l = lambda0 + 85.f * (float)k;
    return l >= 720.f ? l - 340.f : l;
}

// RGB basis b at wavelength l, linear in the staged table (bases: 14 rows of 64)
__device__ inline float basis_value(const float *bases, float l0, float l1, int n, int b, float l) {
    const float x = (l - l0) / (l1 - l0) * (float)(n - 1);
    const float *v = bases + b * 64;
    if (x <= 0.f) return v[0];
    if (x >= (float)(n - 1)) return v[n - 1];
    int j = (int)x;
    if (j > n - 2) j = n - 2;
    const float f = x - (float)j;
    return v[j] * (1.f - f) + v[j + 1] * f;
}
__device__ inline float basis_at(const SmemTables &sm, const TablesArg &t, int b, float l) {
    return basis_value(sm.bases, t.rgb_lambda0, t.rgb_lambda1, t.n_rgb, b, l);
}

__device__ inline float cie_at(const SmemTables &sm, const TablesArg &t, int row, float l) {
    const float x = l - t.cie_lambda0;
    const float *v = sm.cie + row * 512;
    if (x <= 0.f) return v[0];
    if (x >= (float)(t.n_cie - 1)) return v[t.n_cie - 1];
    const int j = (int)x;
    const float f = x - (float)j;
    return v[j] * (1.f - f) + v[j + 1] * f;
}

// from_reflectance_rgb at a hero wavelength from its Smits terms (color/spectrumoperations.cpp:113-147)
__device__ inline float smits_at(const SmemTables &sm, const TablesArg &t, const int basis[3], const float w[3], float l) {
    float r = 0.f;
    for (int k = 0; k < 3; ++k) r += basis_at(sm, t, basis[k], l) * w[k];
    r *= 0.94f;
    return r < 0.f ? 0.f : r;
}

// from_reflectance_rgb at the path's spectral samples
template <int NL>
__device__ inline void reflectance(const SmemTables &sm, const TablesArg &t, const MaterialDev &m,
                                   const float *__restrict__ refl60, float lambda0, Spec<NL> &out) {
    if (NL == 60) {
#pragma unroll 4
        for (int i = 0; i < NL; ++i) out.c[i] = __ldg(refl60 + i);
    } else {
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = smits_at(sm, t, m.basis, m.w, hero_lambda(lambda0, i));
    }
}

// to_xyz (color/spectrumoperations.cpp:193-207), or its hero-wavelength estimator over 380..720 nm
template <int NL>
__device__ inline void spectrum_xyz(const SmemTables &sm, const TablesArg &t, float lambda0, const Spec<NL> &L,
                                    double xyz[3]) {
    float x = 0.f, y = 0.f, z = 0.f;
    if (NL == 60) {
        for (int i = 0; i < NL; ++i) {
            x += sm.binned[i] * L.c[i];
            y += sm.binned[60 + i] * L.c[i];
            z += sm.binned[120 + i] * L.c[i];
        }
        const float scale = (float)(700 - 400) / (float)(t.cie_y_integral * 60);
        xyz[0] = x * scale; xyz[1] = y * scale; xyz[2] = z * scale;
    } else {
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const float l = hero_lambda(lambda0, k);
            x += cie_at(sm, t, 0, l) * L.c[k];
            y += cie_at(sm, t, 1, l) * L.c[k];
            z += cie_at(sm, t, 2, l) * L.c[k];
        }
        const float scale = 340.f / (4.f * t.cie_y_integral);
        xyz[0] = x * scale; xyz[1] = y * scale; xyz[2] = z * scale;
    }
}

// ---------------------------------------------------------------------------- BSDF
// The BSDF and light routines below are called from several places of the shading
// kernels; they are kept out of line (__noinline__) so that each kernel holds one copy:
// fully inlined, the shading kernel overflowed the instruction cache.
template <int NL>
struct Bsdf {
    v3 ng, ns, s, t;
    int type;
    float eta;      // BSDF::eta (etaScale for specular transmission)
    float ax, ay;
    float mat_eta, mat_k;
    Spec<NL> R;
    int corrected;  // FL_RENDER_CORRECTED_GGX: VNDF density and sampling on wo's side
    // FL_MAT_STANDARD: the material record; its colours kd, ks, kt, sheen, coat (in this
    // order) come from the 60-bin table in global memory, or are upsampled at the hero
    // wavelengths when a lobe needs them, from the bases staged in shared memory
    const StandardDev *sd;
    const float *std60;
    const float *bases;
    float rgb_l0, rgb_l1;
    int n_rgb;
    float lambda0;
    int kd_tex;     // kd is an image texture, evaluated at the hit into R
};

enum : int { kStdKd = 0, kStdKs = 1, kStdKt = 2, kStdSheen = 3, kStdCoat = 4, kStdEta = 5, kStdK = 6 };
// the wavelength of spectral sample i: the bin start 400 + 5 i nm (the loop of
// ThinFilmInteference::evaluate) or the hero wavelength
template <int NL>
__device__ inline float std_wavelength(const Bsdf<NL> &b, int i) {
    return NL == 60 ? (float)(400 + 5 * i) : hero_lambda(b.lambda0, i);
}
template <int NL>
__device__ inline float std_color(const Bsdf<NL> &b, int c, int i) {
    if (c == kStdKd && b.kd_tex) return b.R.c[i];
    if (NL == 60) return __ldg(b.std60 + 60 * c + i);
    if (c >= kStdEta) {
        // measured metal: hero wavelengths read the 5 nm bin they fall in, clamped to 400..700 nm
        int bin = (int)floorf((hero_lambda(b.lambda0, i) - 400.f) / 5.f);
        bin = bin < 0 ? 0 : (bin > 59 ? 59 : bin);
        return __ldg(b.std60 + 60 * c + bin);
    }
    // from_reflectance_rgb at hero wavelength i (color/spectrumoperations.cpp:113-147)
    const float l = hero_lambda(b.lambda0, i);
    float r = 0.f;
    for (int k = 0; k < 3; ++k) r += basis_value(b.bases, b.rgb_l0, b.rgb_l1, b.n_rgb, b.sd->basis[c][k], l) * b.sd->w[c][k];
    r *= 0.94f;
    return r < 0.f ? 0.f : r;
}

__device__ inline v3 to_local(v3 s, v3 t, v3 n, v3 v) { return mk(dot(v, s), dot(v, t), dot(v, n)); }
__device__ inline v3 to_world(v3 s, v3 t, v3 n, v3 v) { return add(add(mul(s, v.x), mul(t, v.y)), mul(n, v.z)); }

__device__ inline float cos2t(v3 w) { return w.z * w.z; }
__device__ inline float sin2t(v3 w) { const float v = 1.f - cos2t(w); return v > 0.f ? v : 0.f; }
__device__ inline float sint(v3 w) { return sqrtf(sin2t(w)); }
__device__ inline float tant(v3 w) { return sint(w) / w.z; }
__device__ inline float tan2t(v3 w) { return sin2t(w) / cos2t(w); }
__device__ inline float clampr(float v, float lo, float hi) { if (v < lo) return lo; return v > hi ? hi : v; }
__device__ inline float cosphi(v3 w) { const float st = sint(w); return st == 0.f ? 1.f : clampr(w.x / st, -1.f, 1.f); }
__device__ inline float sinphi(v3 w) { const float st = sint(w); return st == 0.f ? 0.f : clampr(w.y / st, -1.f, 1.f); }
__device__ inline float cos2phi(v3 w) { return cosphi(w) * cosphi(w); }
__device__ inline float sin2phi(v3 w) { return sinphi(w) * sinphi(w); }
__device__ inline bool same_hemi(v3 a, v3 b) { return a.z * b.z > 0; }

template <int NL>
__device__ inline float ggx_D(const Bsdf<NL> &b, v3 wh) {
    const float tan2Theta = tan2t(wh);
    if (isinf(tan2Theta)) return 0.f;
    const float cos4Theta = cos2t(wh) * cos2t(wh);
    const float e = (cos2phi(wh) / (b.ax * b.ax) + sin2phi(wh) / (b.ay * b.ay)) * tan2Theta;
    return 1.f / (kPi * b.ax * b.ay * cos4Theta * (1 + e) * (1 + e));
}
template <int NL>
__device__ inline float ggx_lambda(const Bsdf<NL> &b, v3 w) {
    const float absTanTheta = fabsf(tant(w));
    if (isinf(absTanTheta)) return 0.f;
    const float alpha = sqrtf(cos2phi(w) * b.ax * b.ax + sin2phi(w) * b.ay * b.ay);
    const float a2t2 = (alpha * absTanTheta) * (alpha * absTanTheta);
    return (-1 + sqrtf(1.f + a2t2)) / 2;
}
template <int NL>
__device__ inline float ggx_G(const Bsdf<NL> &b, v3 wo, v3 wi) {
    return 1 / (1 + ggx_lambda(b, wo) + ggx_lambda(b, wi));
}
// Density of the sampled microfacet normal. Reference mode keeps MicrofacetDistribution::pdf
// (microfacet.cpp:14-16), D(wh) |cos theta_h|, although sample_wh draws visible normals
// (quirk Q1). Corrected mode uses the density of the visible normals that sample_wh draws
// (Heitz 2018): G1(wo) |wo . wh| D(wh) / |cos theta_o|.
template <int NL>
__device__ inline float ggx_pdf(const Bsdf<NL> &b, v3 wo, v3 wh) {
    if (b.corrected) {
        if (wo.z == 0.f) return 0.f;
        return ggx_D(b, wh) * absdot(wo, wh) / ((1.f + ggx_lambda(b, wo)) * fabsf(wo.z));
    }
    return ggx_D(b, wh) * fabsf(wh.z);
}
template <int NL>
__device__ inline v3 ggx_sample_wh_upper(const Bsdf<NL> &b, v3 wo, float ux, float uy);
// GGXDistribution::sample_wh (ggx.cpp:32-57): always in the upper hemisphere, even for
// wo.z < 0 (quirk Q2). Corrected mode samples around -wo and flips the normal back to
// wo's side.
template <int NL>
__device__ inline v3 ggx_sample_wh(const Bsdf<NL> &b, v3 wo, float ux, float uy) {
    if (b.corrected && wo.z < 0.f) return neg(ggx_sample_wh_upper(b, neg(wo), ux, uy));
    return ggx_sample_wh_upper(b, wo, ux, uy);
}
template <int NL>
__device__ inline v3 ggx_sample_wh_upper(const Bsdf<NL> &b, v3 wo, float ux, float uy) {
    v3 vh = normalize(mk(wo.x * b.ax, wo.y * b.ay, wo.z));
    if (vh.z < 0) vh = neg(vh);
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const v3 T1 = lensq > 0 ? divs(mk(-vh.y, vh.x, 0.f), sqrtf(lensq)) : mk(1.f, 0.f, 0.f);
    const v3 T2 = cross(vh, T1);
    const float r = sqrtf(ux);
    const float phi = 2.f * kPi * uy;
    const float t1 = r * fl_cos(phi);
    float t2 = r * fl_sin(phi);
    const float s = (float)((1.f + vh.z) * 0.5);
    t2 = (1.f - s) * sqrtf(1 - (t1 * t1)) + (s * t2);
    const float zz = 1.f - t1 * t1 - t2 * t2;
    const v3 Nh = add(add(mul(T1, t1), mul(T2, t2)), mul(vh, sqrtf(zz > 0.f ? zz : 0.f)));
    return normalize(mk(b.ax * Nh.x, b.ay * Nh.y, Nh.z > 1e-6f ? Nh.z : 1e-6f));
}

__device__ inline float fr_dielectric(float cosThetaI, float etaI, float etaT) {
    cosThetaI = clampr(cosThetaI, -1.f, 1.f);
    if (!(cosThetaI > 0.0f)) {
        const float tmp = etaI; etaI = etaT; etaT = tmp;
        cosThetaI = fabsf(cosThetaI);
    }
    const float m = 1.f - cosThetaI * cosThetaI;
    const float sinThetaI = sqrtf(m > 0.f ? m : 0.f);
    const float sinThetaT = etaI / etaT * sinThetaI;
    if (sinThetaT >= 1) return 1.f;
    const float m2 = 1 - sinThetaT * sinThetaT;
    const float cosThetaT = sqrtf(m2 > 0.f ? m2 : 0.f);
    const float Rparl = (etaT * cosThetaI - etaI * cosThetaT) / (etaT * cosThetaI + etaI * cosThetaT);
    const float Rperp = (etaI * cosThetaI - etaT * cosThetaT) / (etaI * cosThetaI + etaT * cosThetaT);
    return (float)((Rparl * Rparl + Rperp * Rperp) * 0.5);
}

__device__ inline float fr_conductor(float cosI, float etaT, float k) {
    cosI = fabsf(cosI);
    cosI = clampr(cosI, -1.f, 1.f);
    const float eta = etaT / 1.f, etak = k / 1.f;
    const float cosThetaI2 = cosI * cosI;
    const float sinThetaI2 = (float)(1. - cosThetaI2);
    const float eta2 = eta * eta, etak2 = etak * etak;
    const float t0 = eta2 - etak2 - sinThetaI2;
    const float a2plusb2 = sqrtf(t0 * t0 + 4.f * eta2 * etak2);
    const float t1 = a2plusb2 + cosThetaI2;
    const float a = sqrtf(0.5f * (a2plusb2 + t0));
    const float t2 = (float)2 * cosI * a;
    const float Rs = (t1 - t2) / (t1 + t2);
    const float t3 = cosThetaI2 * a2plusb2 + sinThetaI2 * sinThetaI2;
    const float t4 = t2 * sinThetaI2;
    const float Rp = Rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (Rp + Rs);
}

// lobes: 0 Lambert, 1 microfacet reflection, 2 microfacet transmission, 3 Fresnel specular,
// and the StandardSurface lobes 4 Oren-Nayar, 5 Fresnel-blended diffuse + specular,
// 6 Estevez sheen, 7 GTR1 clear coat, 8 Fresnel specular with R = ks, T = kt
constexpr int kMaxLobes = 5;
// The BSDF routines are compiled twice: STD = false for the Lambert, GGX and glass
// materials (lobes 0..3), STD = true for the StandardSurface (lobes 4..11) and the
// image-textured Lambert (lobe 0), which the shading kernels' StandardSurface instances
// call. Kept apart, this code adds no calls, registers or branches to the other kernels.
template <bool STD>
__device__ inline int lobe_type(int lobe) {
    if (!STD)
        return lobe == 0 ? (kBsdfReflection | kBsdfDiffuse)
                         : lobe == 1 ? (kBsdfReflection | kBsdfGlossy)
                                     : lobe == 2 ? (kBsdfTransmission | kBsdfGlossy)
                                                 : (kBsdfReflection | kBsdfTransmission | kBsdfSpecular);
    return (lobe == 0 || lobe == 4) ? (kBsdfReflection | kBsdfDiffuse)
                     : lobe == 11 ? (kBsdfTransmission | kBsdfDiffuse)
                                  : lobe == 8 ? (kBsdfReflection | kBsdfTransmission | kBsdfSpecular)
                                              : (kBsdfReflection | kBsdfGlossy);
}
template <bool STD, int NL>
__device__ inline int mat_lobes(const Bsdf<NL> &b, int *lobes) {
    if (STD) {
        if (b.type == FL_MAT_LAMBERT) { lobes[0] = 0; return 1; }  // image-textured Lambert
#pragma unroll
        for (int i = 0; i < kMaxLobes; ++i) lobes[i] = b.sd->lobes[i];
        return b.sd->n_lobes;
    }
    switch (b.type) {
    case FL_MAT_LAMBERT: lobes[0] = 0; return 1;
    case FL_MAT_CONDUCTOR: lobes[0] = 1; return 1;
    case FL_MAT_ROUGH_DIELECTRIC: lobes[0] = 1; lobes[1] = 2; return 2;
    default: lobes[0] = 3; return 1;
    }
}

// ---- StandardSurface lobe helpers
// OrenNayarBRDF::OrenNayarBRDF / evaluate (bxdfs/orennayar.cpp:6-39); A, B precomputed per material
template <int NL>
__device__ inline void oren_nayar_eval(const Bsdf<NL> &b, float A, float B, v3 wo, v3 wi, Spec<NL> &out) {
    const float sinThetaI = sint(wi), sinThetaO = sint(wo);
    float maxCos = 0.f;
    if (sinThetaI > 1e-4 && sinThetaO > 1e-4) {
        const float sinPhiI = sinphi(wi), cosPhiI = cosphi(wi), sinPhiO = sinphi(wo), cosPhiO = cosphi(wo);
        const float dCos = cosPhiI * cosPhiO + sinPhiI * sinPhiO;
        maxCos = dCos > 0.f ? dCos : 0.f;
    }
    float sinAlpha, tanBeta;
    if (fabsf(wi.z) > fabsf(wo.z)) { sinAlpha = sinThetaO; tanBeta = sinThetaI / fabsf(wi.z); }
    else { sinAlpha = sinThetaI; tanBeta = sinThetaO / fabsf(wo.z); }
    const float v = (A + B * maxCos * sinAlpha * tanBeta);
    const float weight = b.sd->kd_weight;
#pragma unroll
    for (int i = 0; i < NL; ++i) out.c[i] = std_color(b, kStdKd, i) * kInvPi * v * weight;
}
// concentric_sample_disk (core/shadingcore.h:65-80), as (x, y, 0)
__device__ inline v3 concentric_disk(float ux, float uy) {
    const float ox = ux * 2.f - 1.f, oy = uy * 2.f - 1.f;
    if (ox == 0 && oy == 0) return mk(0.f, 0.f, 0.f);
    float theta, r;
    if (fabsf(ox) > fabsf(oy)) { r = ox; theta = kPiOver4 * (oy / ox); }
    else { r = oy; theta = kPiOver2 - kPiOver4 * (ox / oy); }
    return mk(r * fl_cos(theta), r * fl_sin(theta), 0.f);
}
// cosine_hemisphere_sample over concentric_sample_disk (core/shadingcore.h:65-89), on wo's side
__device__ inline v3 cos_hemi(v3 wo, float ux, float uy) {
    const v3 dsk = concentric_disk(ux, uy);
    const float dx = dsk.x, dy = dsk.y;
    const float zz = 1.f - dx * dx - dy * dy;
    v3 wi = mk(dx, dy, sqrtf(zz > 0.f ? zz : 0.f));
    if (wo.z < 0) wi.z *= -1.f;
    return wi;
}
__device__ inline v3 reflect_wh(v3 wo, v3 wh) { return sub(mul(mul(wh, 2.f), dot(wo, wh)), wo); }
// EstevezSheenDistribution D and Lambda (microfacets/estevez.cpp:11-34)
__device__ inline float est_D(float r, v3 wh) {
    const float inv = 1.f / r;
    return (2.f + inv) * fl_pow(sint(wh), inv) / (2.f * kPi);
}
__device__ inline float est_plerp(float r, float p0, float p1) {
    return ((1.f - r) * (1.f - r)) * p0 + (1.f - ((1.f - r) * (1.f - r))) * p1;
}
__device__ inline float est_lambda(float r, v3 w) {
    const float a = est_plerp(r, 25.3245f, 21.5473f), b = est_plerp(r, 3.32435f, 3.82987f);
    const float c = est_plerp(r, 0.16801f, 0.19823f), d = est_plerp(r, -1.27393f, -1.97760f);
    const float e = est_plerp(r, -4.85967f, -4.32054f);
    auto L = [&](float v) { return a / (1.f + b * fl_pow(v, c)) + (d * v) + e; };
    const float ac = fabsf(w.z);
    if (ac < 0.5f) return fl_exp(L(ac));
    return fl_exp(2.f * L(0.5f) - L(1.f - ac));
}
// ClearcoatReflectionBRDF's GTR1 and Smith G (bxdfs/clearcoat.cpp:8-19). The reference's
// smithG_GGX calls the unqualified sqrt, the double-precision C function, so the parity
// build carries that sum and division in double.
__device__ inline float gtr1(float cosTheta, float alpha) {
    const float alpha2 = alpha * alpha;
    return (alpha2 - 1) / (kPi * fl_log(alpha2) * (1 + (alpha2 - 1) * cosTheta * cosTheta));
}
__device__ inline float smith_g_ggx(float cosTheta, float alpha) {
    const float alpha2 = alpha * alpha, cosTheta2 = cosTheta * cosTheta;
#if defined(FL_PARITY_MATH)
    return (float)(1.f / ((double)cosTheta + sqrt((double)(alpha2 + cosTheta2 - alpha2 * cosTheta2))));
#else
    return 1.f / (cosTheta + sqrtf(alpha2 + cosTheta2 - alpha2 * cosTheta2));
#endif
}
__device__ inline bool matches(int type, int flags) { return (type & flags) == type; }

// ThinFilmInteference::evaluate (fresnel/thinfilm.cpp:8-58) with extIOR 1 and the amplitude
// coefficients of fresnel/fresnel.h:9-23, at the path's wavelengths. The reference's sin^2
// ratios divide a quotient by itself, so both equal 1 - cos^2 (kept).
template <int NL>
__device__ inline void thin_film_fresnel(const Bsdf<NL> &b, float cosThetaI, Spec<NL> &F) {
    const float extIOR = 1.f, tfIOR = b.sd->tf_ior, mIOR = b.mat_eta, thickness = b.sd->tf_thickness;
    const float sinSqrd1 = ((extIOR / tfIOR) / (extIOR / tfIOR)) * (1 - cosThetaI * cosThetaI);
    const float sinSqrd2 = ((extIOR / mIOR) / (extIOR / mIOR)) * (1 - cosThetaI * cosThetaI);
    if ((sinSqrd1 > 1) || (sinSqrd2 > 1)) { F.set(1.f); return; }
    const float cos1 = sqrtf(1 - sinSqrd1);
    const float cos2 = sqrtf(1 - sinSqrd2);
    auto sp_r = [](float n1, float n2, float ci, float ct) { return (n1 * ci - n2 * ct) / (n1 * ci + n2 * ct); };
    auto sp_t = [](float n1, float n2, float ci, float ct) { return (2.f * n1 * ci) / (n1 * ci + n2 * ct); };
    auto pp_r = [](float n1, float n2, float ci, float ct) { return (n2 * ci - n1 * ct) / (n1 * ct + n2 * ci); };
    auto pp_t = [](float n1, float n2, float ci, float ct) { return (2.f * n1 * ci) / (n1 * ct + n2 * ci); };
    const float alphaSP = sp_r(tfIOR, extIOR, cos1, cosThetaI) * sp_r(mIOR, tfIOR, cos1, cos2);
    const float alphaPP = pp_r(tfIOR, extIOR, cos1, cosThetaI) * pp_r(mIOR, tfIOR, cos1, cos2);
    const float betaSP = sp_t(extIOR, tfIOR, cosThetaI, cos1) * sp_t(tfIOR, mIOR, cos1, cos2);
    const float betaPP = pp_t(extIOR, tfIOR, cosThetaI, cos1) * pp_t(tfIOR, mIOR, cos1, cos2);
    const float delta10 = tfIOR < extIOR ? kPi : 0.f;
    const float delta12 = tfIOR < mIOR ? kPi : 0.f;
    const float delta = delta10 + delta12;
    const float beamRatio = (mIOR * cos2) / (extIOR * cosThetaI);
    for (int i = 0; i < NL; ++i) {
        const float wavelength = std_wavelength(b, i);
        const float phi = (2.f * kPi / wavelength) * (2.f * tfIOR * thickness * cos1) + delta;
        const float cp = fl_cos(phi);
        const float ts = (betaSP * betaSP) / ((alphaSP * alphaSP) - (2.f * alphaSP * cp) + 1.f);
        const float tp = (betaPP * betaPP) / ((alphaPP * alphaPP) - (2.f * alphaPP * cp) + 1.f);
        F.c[i] = 1.f - (ts + tp) * 0.5f * beamRatio;
    }
}

// StandardSurface lobes 4..7 and 9..11, out of line: they are the rarely run part of the shading
// kernels, and kept apart their registers do not weigh on the Lambert and GGX code.
template <int NL>
__device__ __noinline__ void std_lobe_eval(const Bsdf<NL> &b, int lobe, v3 wo, v3 wi, Spec<NL> &out) {
    if (lobe == 4) { oren_nayar_eval(b, b.sd->on_A, b.sd->on_B, wo, wi, out); return; }
    if (lobe == 5) {
        // FresnelBlendedDiffuseSpecularBRDF::evaluate (closures/fresnelblendeddiffspec.cpp:18-38)
        const StandardDev &sd = *b.sd;
        const float r1 = 1.f - .5f * fabsf(wi.z);
        const float r1pow5 = (r1 * r1) * (r1 * r1) * r1;
        const float r2 = 1.f - .5f * fabsf(wo.z);
        const float r2pow5 = (r2 * r2) * (r2 * r2) * r2;
        v3 wh = add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) { out.set(0.f); return; }
        oren_nayar_eval(b, sd.fb_A, sd.fb_B, wo, wi, out);
        wh = normalize(wh);
        const float cF = dot(wi, wh);
        const float D = ggx_D(b, wh);
        const float den = (4.f * absdot(wi, wh) * fmaxf(fabsf(wi.z), fabsf(wo.z)));
        const float R1 = 1.f - cF;
        const float ro = sd.ro, ksw = sd.ks_weight;
        const bool metallic = sd.fresnel_type == FL_FRESNEL_METALLIC;
        const float r1p5 = metallic ? (R1 * R1 * R1 * R1 * R1) : ((R1 * R1) * (R1 * R1) * R1);
#pragma unroll
        for (int i = 0; i < NL; ++i) {
            const float diffuse = (28.f / 23.f) * out.c[i] * (1.f - ro) * (1 - r1pow5) * (1 - r2pow5);
            const float ks = std_color(b, kStdKs, i);
            // SchlickMetallic (r0 = ks, fresnel/schlickmetallic.cpp:7-10) or SchlickDielectric
            // (fresnel/schlickdielectric.cpp:7-11)
            const float F = metallic ? ks + (1.f - ks) * r1p5 : ro + r1p5 * (1.f - ro);
            float specular = D * F / den;
            specular = ks * specular * ksw;
            out.c[i] = diffuse + specular;
        }
        return;
    }
    if (lobe == 6) {
        // MicrofacetReflectionBRDF::evaluate with the Estevez distribution and FresnelNull
        const float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { out.set(0.f); return; }
        wh = normalize(wh);
        const float r = b.sd->sheen_rough, w = b.sd->sheen_weight;
        const float D = est_D(r, wh);
        const float G = 1.f / (1.f + est_lambda(r, wo) + est_lambda(r, wi));
        const float den = 4.f * cosThetaO * cosThetaI;
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = std_color(b, kStdSheen, i) * w * D * G * 1.f / den;
        return;
    }
    if (lobe == 7) {
        // ClearcoatReflectionBRDF::evaluate (bxdfs/clearcoat.cpp:28-41)
        v3 wh = add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) { out.set(0.f); return; }
        wh = normalize(wh);
        const float Dr = gtr1(fabsf(wh.z), b.sd->coat_gloss);
        const float Fr = fr_dielectric(dot(wo, wh), 1.f, b.sd->coat_ior);
        const float Gr = smith_g_ggx(fabsf(wo.z), .25f) * smith_g_ggx(fabsf(wi.z), .25f);
        const float w = b.sd->coat_weight;
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = std_color(b, kStdCoat, i) * Fr * w * Gr * Dr / 4;
        return;
    }
    if (lobe == 9 || lobe == 10) {
        // MicrofacetReflectionBRDF::evaluate (bxdfs/microfacetreflection.cpp:13-32) with R = 1 and
        // the measured-metal FresnelConductor (weight ks_weight) or the thin film (weight 1)
        const float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { out.set(0.f); return; }
        wh = normalize(wh);
        const v3 whf = dot(wh, mk(0.f, 0.f, 1.f)) < 0.f ? neg(wh) : wh;
        const float cF = dot(wi, whf);
        if (lobe == 9) {
#pragma unroll 4
            for (int i = 0; i < NL; ++i) out.c[i] = fr_conductor(cF, std_color(b, kStdEta, i), std_color(b, kStdK, i));
        } else {
            thin_film_fresnel(b, cF, out);
        }
        const float weight = lobe == 9 ? b.sd->ks_weight : 1.f;
        const float D = ggx_D(b, wh), G = ggx_G(b, wo, wi);
        const float den = 4.f * cosThetaO * cosThetaI;
#pragma unroll 4
        for (int i = 0; i < NL; ++i) out.c[i] = 1.f * weight * D * G * out.c[i] / den;
        return;
    }
    if (lobe == 11) { oren_nayar_eval(b, b.sd->on_A, b.sd->on_B, wo, wi, out); return; }
    out.set(0.f);
}

template <int NL>
__device__ __noinline__ float std_lobe_pdf(const Bsdf<NL> &b, int lobe, v3 wo, v3 wi) {
    if (lobe == 4) return same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.f;
    if (lobe == 5) {
        // closures/fresnelblendeddiffspec.cpp:61-67
        if (!same_hemi(wo, wi)) return 0.f;
        const v3 wh = normalize(add(wo, wi));
        const float pdf_wh = ggx_pdf(b, wo, wh);
        return .5f * (fabsf(wi.z) * kInvPi + pdf_wh / (4 * dot(wo, wh)));
    }
    if (lobe == 6) {
        // MicrofacetReflectionBRDF::pdf with MicrofacetDistribution::pdf = D |cos theta_h|
        if (!same_hemi(wo, wi)) return 0.f;
        const v3 wh = normalize(add(wo, wi));
        return est_D(b.sd->sheen_rough, wh) * fabsf(wh.z) / (4.f * dot(wo, wh));
    }
    if (lobe == 7) {
        // bxdfs/clearcoat.cpp:70-80
        if (!same_hemi(wo, wi)) return 0.f;
        v3 wh = add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) return 0.f;
        wh = normalize(wh);
        const float Dr = gtr1(fabsf(wh.z), b.sd->coat_gloss);
        return Dr * fabsf(wh.z) / (4 * dot(wo, wh));
    }
    if (lobe == 9 || lobe == 10) {
        if (!same_hemi(wo, wi)) return 0.f;
        const v3 wh = normalize(add(wo, wi));
        return ggx_pdf(b, wo, wh) / (4.f * dot(wo, wh));
    }
    // DiffuseTransmission::pdf (bxdfs/diffusetransmission.cpp:29-31)
    if (lobe == 11) return !same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.f;
    return 0.f;
}

template <int NL>
__device__ __noinline__ void std_lobe_sample(const Bsdf<NL> &b, int lobe, v3 wo, v3 &wi, float ux, float uy, float &pdf,
                                             Spec<NL> &f) {
    if (lobe == 4) {
        // OrenNayarBRDF::sample (bxdfs/orennayar.cpp:41-56): a cosine-weighted direction on wo's side
        wi = cos_hemi(wo, ux, uy);
        pdf = std_lobe_pdf(b, 4, wo, wi);
        std_lobe_eval(b, 4, wo, wi, f);
        return;
    }
    if (lobe == 5) {
        // FresnelBlendedDiffuseSpecularBRDF::sample (closures/fresnelblendeddiffspec.cpp:40-59)
        if (ux < .5) {
            float u0 = 2 * ux;
            if (u0 > 1.f - kShadowEpsilon) u0 = 1.f - kShadowEpsilon;
            wi = cos_hemi(wo, u0, uy);
        } else {
            float u0 = 2 * (ux - .5f);
            if (u0 > 1.f - kShadowEpsilon) u0 = 1.f - kShadowEpsilon;
            wi = reflect_wh(wo, ggx_sample_wh(b, wo, u0, uy));
            if (!same_hemi(wo, wi)) { f.set(0.f); return; }
        }
        pdf = std_lobe_pdf(b, 5, wo, wi);
        std_lobe_eval(b, 5, wo, wi, f);
        return;
    }
    if (lobe == 6) {
        // MicrofacetReflectionBRDF::sample (bxdfs/microfacetreflection.cpp:30-52); the Estevez
        // sample_wh is a cosine-weighted normal on wo's side (microfacets/estevez.cpp:36-42)
        if (wo.z == 0) { f.set(0.f); return; }
        const v3 wh = cos_hemi(wo, ux, uy);
        if (dot(wo, wh) < 0) { f.set(0.f); return; }
        wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, wi)) { f.set(0.f); return; }
        pdf = est_D(b.sd->sheen_rough, wh) * fabsf(wh.z) / (4.f * dot(wo, wh));
        std_lobe_eval(b, 6, wo, wi, f);
        return;
    }
    if (lobe == 7) {
        // ClearcoatReflectionBRDF::sample (bxdfs/clearcoat.cpp:43-68)
        if (wo.z == 0) { f.set(0.f); return; }
        const float g = b.sd->coat_gloss;
        const float alpha2 = g * g;
        const float cosTheta = sqrtf(fmaxf(0.f, (1 - fl_pow(alpha2, 1 - ux)) / (1 - alpha2)));
        const float sinTheta = sqrtf(fmaxf(0.f, 1 - cosTheta * cosTheta));
        const float phi = 2 * kPi * uy;
        v3 wh = mk(sinTheta * fl_cos(phi), sinTheta * fl_sin(phi), cosTheta);
        if (!same_hemi(wo, wh)) wh = neg(wh);
        wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, wi)) { f.set(0.f); return; }
        pdf = std_lobe_pdf(b, 7, wo, wi);
        std_lobe_eval(b, 7, wo, wi, f);
        return;
    }
    if (lobe == 9 || lobe == 10) {
        // MicrofacetReflectionBRDF::sample (bxdfs/microfacetreflection.cpp:34-56)
        if (wo.z == 0) { f.set(0.f); return; }
        const v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (dot(wo, wh) < 0) { f.set(0.f); return; }
        wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, wi)) { f.set(0.f); return; }
        pdf = ggx_pdf(b, wo, wh) / (4.f * dot(wo, wh));
        std_lobe_eval(b, lobe, wo, wi, f);
        return;
    }
    if (lobe == 11) {
        // DiffuseTransmission::sample (bxdfs/diffusetransmission.cpp:16-27): a cosine-weighted
        // direction on the side away from wo
        wi = cos_hemi(mk(0.f, 0.f, 1.f), ux, uy);
        if (wo.z > 0) wi.z *= -1.f;
        pdf = std_lobe_pdf(b, 11, wo, wi);
        std_lobe_eval(b, 11, wo, wi, f);
        return;
    }
    f.set(0.f);
}

// lobe evaluate into out (reference multiplication order)
template <bool STD, int NL>
__device__ inline void lobe_eval(const Bsdf<NL> &b, int lobe, v3 wo, v3 wi, Spec<NL> &out) {
    if (STD && lobe != 0) {
        if (lobe != 8) std_lobe_eval(b, lobe, wo, wi, out);
        else out.set(0.f);
        return;
    }
    if (lobe == 0) {
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = b.R.c[i] * kInvPi * 1.f;
        return;
    }
    if (lobe == 1) {
        const float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { out.set(0.f); return; }
        wh = normalize(wh);
        const v3 whf = dot(wh, mk(0.f, 0.f, 1.f)) < 0.f ? neg(wh) : wh;
        const float cF = dot(wi, whf);
        const float F = b.type == FL_MAT_CONDUCTOR ? fr_conductor(cF, b.mat_eta, b.mat_k) : fr_dielectric(cF, 1.f, b.mat_eta);
        const float D = ggx_D(b, wh), G = ggx_G(b, wo, wi);
        const float den = 4.f * cosThetaO * cosThetaI;
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = b.R.c[i] * 1.f * D * G * F / den;
        return;
    }
    if (lobe == 2) {
        if (same_hemi(wo, wi)) { out.set(0.f); return; }
        const float cosThetaO = wo.z, cosThetaI = wi.z;
        if (cosThetaI == 0 || cosThetaO == 0) { out.set(0.f); return; }
        const float eta = wo.z > 0 ? (b.mat_eta / 1.f) : (1.f / b.mat_eta);
        v3 wh = normalize(add(wo, mul(wi, eta)));
        if (wh.z < 0) wh = neg(wh);
        if (dot(wo, wh) * dot(wi, wh) > 0) { out.set(0.f); return; }
        const float F = fr_dielectric(dot(wo, wh), 1.f, b.mat_eta);
        const float sqrtDenom = dot(wo, wh) + eta * dot(wi, wh);
        const float factor = (1 / eta);
        const float v = fabsf(ggx_D(b, wh) * ggx_G(b, wo, wi) * eta * eta * absdot(wi, wh) * absdot(wo, wh) * factor *
                              factor / (cosThetaI * cosThetaO * sqrtDenom * sqrtDenom));
#pragma unroll
        for (int i = 0; i < NL; ++i) out.c[i] = (1.f - F) * b.R.c[i] * v;
        return;
    }
    out.set(0.f);
}

template <bool STD, int NL>
__device__ inline float lobe_pdf(const Bsdf<NL> &b, int lobe, v3 wo, v3 wi) {
    if (STD && lobe != 0) return lobe != 8 ? std_lobe_pdf(b, lobe, wo, wi) : 0.f;
    if (lobe == 0) return same_hemi(wo, wi) ? fabsf(wi.z) * kInvPi : 0.f;
    if (lobe == 1) {
        if (!same_hemi(wo, wi)) return 0.f;
        const v3 wh = normalize(add(wo, wi));
        return ggx_pdf(b, wo, wh) / (4.f * dot(wo, wh));
    }
    if (lobe == 2) {
        if (same_hemi(wo, wi)) return 0.f;
        const float eta = wo.z > 0 ? (b.mat_eta / 1.f) : (1.f / b.mat_eta);
        const v3 wh = normalize(add(wo, mul(wi, eta)));
        if (dot(wo, wh) * dot(wi, wh) > 0) return 0.f;
        const float sqrtDenom = dot(wo, wh) + eta * dot(wi, wh);
        const float dwh_dwi = fabsf((eta * eta * dot(wi, wh)) / (sqrtDenom * sqrtDenom));
        return ggx_pdf(b, wo, wh) * dwh_dwi;
    }
    return 0.f;
}

template <bool STD, int NL>
__device__ inline void lobe_sample(const Bsdf<NL> &b, int lobe, v3 wo, v3 &wi, float ux, float uy, float &pdf,
                                   int &type, Spec<NL> &f) {
    if (lobe == 0) {
        // LambertBRDF::sample: a cosine-weighted direction on wo's side
        wi = cos_hemi(wo, ux, uy);
        pdf = lobe_pdf<false>(b, 0, wo, wi);
        lobe_eval<false>(b, 0, wo, wi, f);
        return;
    }
    if (lobe == 1) {
        if (wo.z == 0) { f.set(0.f); return; }
        const v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (dot(wo, wh) < 0) { f.set(0.f); return; }
        wi = sub(mul(mul(wh, 2.f), dot(wo, wh)), wo);
        if (!same_hemi(wo, wi)) { f.set(0.f); return; }
        pdf = ggx_pdf(b, wo, wh) / (4.f * dot(wo, wh));
        lobe_eval<false>(b, 1, wo, wi, f);
        return;
    }
    if (lobe == 2) {
        if (wo.z == 0) { f.set(0.f); return; }
        const v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (dot(wo, wh) < 0) { f.set(0.f); return; }
        const float eta = wo.z > 0 ? (1.f / b.mat_eta) : (b.mat_eta / 1.f);
        const float cosI = dot(wo, wh);
        const float m = 1.f - (cosI * cosI);
        const float sinI2 = m > 0.f ? m : 0.f;
        const float sinT2 = eta * eta * sinI2;
        if (sinT2 >= 1) { f.set(0.f); return; }
        const float cosT = sqrtf(1 - sinT2);
        wi = add(mul(wo, -eta), mul(wh, (eta * cosI - cosT)));
        pdf = lobe_pdf<false>(b, 2, wo, wi);
        lobe_eval<false>(b, 2, wo, wi, f);
        return;
    }
    if (STD && lobe != 8) { std_lobe_sample(b, lobe, wo, wi, ux, uy, pdf, f); return; }
    // FresnelSpecularBXDF: lobe 3 with R = T = the material colour, lobe 8 with R = ks, T = kt
    const float F = fr_dielectric(wo.z, 1.f, b.mat_eta);
    if (ux < F) {
        wi = mk(-wo.x, -wo.y, wo.z);
        type = kBsdfSpecular | kBsdfReflection;
        pdf = F;
        const float ac = fabsf(wi.z);
#pragma unroll
        for (int i = 0; i < NL; ++i) f.c[i] = (STD ? std_color(b, kStdKs, i) : b.R.c[i]) * F / ac;
    } else {
        const bool entering = wo.z > 0;
        const float etaI = entering ? 1.f : b.mat_eta;
        const float etaT = entering ? b.mat_eta : 1.f;
        const v3 n = dot(mk(0.f, 0.f, 1.f), wo) < 0.f ? mk(-0.f, -0.f, -1.f) : mk(0.f, 0.f, 1.f);
        const float eta = etaI / etaT;
        const float cosI = dot(wo, n);
        const float m = 1.f - (cosI * cosI);
        const float sinI2 = m > 0.f ? m : 0.f;
        const float sinT2 = eta * eta * sinI2;
        if (sinT2 >= 1) { f.set(0.f); return; }
        const float cosT = sqrtf(1 - sinT2);
        wi = add(mul(wo, -eta), mul(n, (eta * cosI - cosT)));
        const float sc = (etaI * etaI) / (etaT * etaT);
        type = kBsdfSpecular | kBsdfTransmission;
        pdf = 1.f - F;
        const float ac = fabsf(wi.z);
#pragma unroll
        for (int i = 0; i < NL; ++i) {
            float ft = (STD ? std_color(b, kStdKt, i) : b.R.c[i]) * (1.f - F);
            ft *= sc;
            f.c[i] = ft / ac;
        }
    }
}

template <bool STD, int NL>
__device__ inline int bsdf_num_components(const Bsdf<NL> &b, int flags) {
    int lobes[kMaxLobes];
    const int n = mat_lobes<STD>(b, lobes);
    int c = 0;
    for (int i = 0; i < n; ++i) c += matches(lobe_type<STD>(lobes[i]), flags) ? 1 : 0;
    return c;
}

template <bool STD, int NL>
__device__ __noinline__ void bsdf_eval(const Bsdf<NL> &b, v3 woW, v3 wiW, int flags, Spec<NL> &out) {
    const v3 wi = to_local(b.s, b.t, b.ns, wiW), wo = to_local(b.s, b.t, b.ns, woW);
    out.set(0.f);
    if (wo.z == 0) return;
    const bool reflect = dot(wiW, b.ng) * dot(woW, b.ng) > 0;
    int lobes[kMaxLobes];
    const int n = mat_lobes<STD>(b, lobes);
    for (int i = 0; i < n; ++i) {
        const int ty = lobe_type<STD>(lobes[i]);
        if (matches(ty, flags) && ((reflect && (ty & kBsdfReflection)) || (!reflect && (ty & kBsdfTransmission)))) {
            Spec<NL> f;
            lobe_eval<STD>(b, lobes[i], wo, wi, f);
#pragma unroll
            for (int k = 0; k < NL; ++k) out.c[k] += f.c[k];
        }
    }
}

template <bool STD, int NL>
__device__ __noinline__ float bsdf_pdf(const Bsdf<NL> &b, v3 woW, v3 wiW, int flags) {
    int lobes[kMaxLobes];
    const int n = mat_lobes<STD>(b, lobes);
    const v3 wi = to_local(b.s, b.t, b.ns, wiW), wo = to_local(b.s, b.t, b.ns, woW);
    if (wo.z == 0) return 0.f;
    float pdf = 0.f;
    int mc = 0;
    for (int i = 0; i < n; ++i)
        if (matches(lobe_type<STD>(lobes[i]), flags)) { ++mc; pdf += lobe_pdf<STD>(b, lobes[i], wo, wi); }
    return mc > 0 ? pdf / (float)mc : 0.f;
}

template <bool STD, int NL>
__device__ __noinline__ void bsdf_sample(const Bsdf<NL> &b, v3 woW, v3 &wiW, float ux, float uy, float &pdf, int flags,
                                   int &sampledType, Spec<NL> &f) {
    int lobes[kMaxLobes];
    const int n = mat_lobes<STD>(b, lobes);
    int mc = 0;
    for (int i = 0; i < n; ++i) mc += matches(lobe_type<STD>(lobes[i]), flags) ? 1 : 0;
    f.set(0.f);
    if (mc == 0) { pdf = 0.f; sampledType = 0; return; }
    int comp = (int)floorf(ux * mc);
    if (comp > mc - 1) comp = mc - 1;
    int chosen = lobes[0], count = comp;
    for (int i = 0; i < n; ++i)
        if (matches(lobe_type<STD>(lobes[i]), flags) && count-- == 0) { chosen = lobes[i]; break; }
    float urx = ux * mc - comp;
    if (urx > 1.f - kShadowEpsilon) urx = 1.f - kShadowEpsilon;
    v3 wi = mk(0.f, 0.f, 0.f);
    const v3 wo = to_local(b.s, b.t, b.ns, woW);
    if (wo.z == 0) return;
    pdf = 0.f;
    const int ctype = lobe_type<STD>(chosen);
    sampledType = ctype;
    lobe_sample<STD>(b, chosen, wo, wi, urx, uy, pdf, sampledType, f);
    if (pdf == 0) { sampledType = 0; f.set(0.f); return; }
    wiW = to_world(b.s, b.t, b.ns, wi);
    if (!(ctype & kBsdfSpecular) && mc > 1) {
        for (int i = 0; i < n; ++i)
            if (lobes[i] != chosen && matches(lobe_type<STD>(lobes[i]), flags)) pdf += lobe_pdf<STD>(b, lobes[i], wo, wi);
    }
    if (mc > 1) pdf /= mc;
    if (!(ctype & kBsdfSpecular)) {
        const bool reflect = dot(wiW, b.ng) * dot(woW, b.ng) > 0;
        f.set(0.f);
        for (int i = 0; i < n; ++i) {
            const int ty = lobe_type<STD>(lobes[i]);
            if (matches(ty, flags) && ((reflect && (ty & kBsdfReflection)) || (!reflect && (ty & kBsdfTransmission)))) {
                Spec<NL> g;
                lobe_eval<STD>(b, lobes[i], wo, wi, g);
#pragma unroll
                for (int k = 0; k < NL; ++k) f.c[k] += g.c[k];
            }
        }
    }
}

// ---------------------------------------------------------------------------- geometry
struct Hit {
    v3 p, n, wo;   // pError is 0 for every hit (BVH::intersect computes gamma<int>(5) == 0)
    int prim;      // triangle id, or -2 - light for a sphere light
    float b1, b2;  // barycentrics of the triangle's second and third vertex
};

// offset_point_origin (core/interaction.h:11-31) with pError = 0: the origin is p itself
// apart from the sign of zero terms, which p + (+-0) keeps.
__device__ inline v3 spawn_origin(v3 p, v3 n, v3 w) {
    v3 offset = mul(n, 0.f);
    if (dot(w, n) < 0) offset = neg(offset);
    return add(p, offset);
}

__device__ inline v3 tri_v(const float *__restrict__ soup, uint32_t id, int k) {
    const float *v = soup + 9 * (size_t)id + 3 * k;
    return mk(__ldg(v), __ldg(v + 1), __ldg(v + 2));
}

// Triangle::intersect (triangle.cpp:13-124), used by Shape::pdf for one light triangle
__device__ inline bool tri_intersect_ref(v3 v1, v3 v2, v3 v3v, v3 ro, v3 rd, float tmin, float tmax, v3 &p, v3 &n) {
    const v3 e1 = sub(v2, v1), e2 = sub(v3v, v1);
    const v3 nn = cross(e1, e2);
    const float det = -dot(rd, nn);
    const v3 ao = sub(ro, v1);
    const v3 dao = cross(ao, rd);
    const float invDet = FL_DIV(1.f, det);
    const float alpha = FL_MUL(dot(e2, dao), invDet);
    const float beta = FL_MUL(-dot(e1, dao), invDet);
    const float t = FL_MUL(dot(ao, nn), invDet);
    if ((t < tmax && t > tmin) && alpha > 0 && beta > 0 && FL_ADD(alpha, beta) < 1.f) {
        if (len2(nn) == 0) return false;
        p = add(ro, mul(rd, t));
        n = normalize(cross(sub(v1, v3v), sub(v2, v3v)));
        return true;
    }
    return false;
}

__device__ inline float sphere_hit(const LightDev &L, v3 o, v3 d, float tmin, float tmax) {
    const v3 oc = sub(o, mk(L.cx, L.cy, L.cz));
    const float a = dot(d, d);
    const float b = dot(oc, d);
    const float cc = dot(oc, oc) - L.radius * L.radius;
    const float disc = b * b - a * cc;
    if (disc < 0.f || a == 0.f) return -1.f;
    const float sq = sqrtf(disc);
    const float t0 = (-b - sq) / a, t1 = (-b + sq) / a;
    if (t0 > tmin && t0 < tmax) return t0;
    if (t1 > tmin && t1 < tmax) return t1;
    return -1.f;
}

struct LightSample {
    v3 wi;
    float pdf;
    float radiance;
    int vis_kind;  // 1: segment to target, 2: direction to infinity
    v3 target;
};

// Illuminant::sample_li for the three light types
static __device__ __noinline__ LightSample light_sample_li(const LightDev &L, const float *__restrict__ soup, const Hit &ref,
                                              float ux, float uy) {
    LightSample ls;
    ls.pdf = 0.f;
    ls.radiance = 0.f;
    ls.vis_kind = 0;
    ls.wi = mk(0.f, 0.f, 0.f);
    ls.target = mk(0.f, 0.f, 0.f);
    if (L.type == FL_LIGHT_TRIANGLE) {
        const v3 p0 = tri_v(soup, L.tri, 0), p1 = tri_v(soup, L.tri, 1), p2 = tri_v(soup, L.tri, 2);
        const float uu = sqrtf(ux);
        const float u1 = 1.f - uu;
        const float u2 = uy * uu;
        const v3 ip = add(add(mul(p0, u1), mul(p1, u2)), mul(p2, (1.f - u1 - u2)));
        const v3 in = normalize(cross(sub(p1, p0), sub(p2, p0)));
        float pdf = 1.f / L.area;
        v3 w = sub(ip, ref.p);
        if (len2(w) == 0) pdf = 0.f;
        else {
            w = normalize(w);
            pdf *= len2(sub(ref.p, ip)) / absdot(in, neg(w));
            if (isinf(pdf)) pdf = 0.f;
        }
        if (pdf == 0 || len2(sub(ip, ref.p)) == 0) return ls;
        ls.pdf = pdf;
        ls.wi = normalize(sub(ip, ref.p));
        ls.vis_kind = 1;
        ls.target = ip;
        ls.radiance = dot(in, mk(-ls.wi.x, -ls.wi.y, -ls.wi.z)) > 0.f ? L.radiance : 0.f;
        return ls;
    }
    if (L.type == FL_LIGHT_SPHERE) {
        const v3 c = mk(L.cx, L.cy, L.cz);
        const float z = 1.f - 2.f * ux;
        const float rr = sqrtf(fmaxf(0.f, 1.f - z * z));
        const float phi = 2.f * kPi * uy;
        const v3 nrm = mk(rr * fl_cos(phi), rr * fl_sin(phi), z);
        const v3 ip = add(c, mul(nrm, L.radius));
        v3 w = sub(ip, ref.p);
        const float d2 = len2(w);
        if (d2 == 0) return ls;
        w = normalize(w);
        const float cosl = dot(nrm, neg(w));
        if (cosl <= 0.f) return ls;
        const float pdf = d2 / (cosl * L.area);
        if (isinf(pdf)) return ls;
        ls.pdf = pdf;
        ls.wi = w;
        ls.vis_kind = 1;
        ls.target = ip;
        ls.radiance = L.radiance;
        return ls;
    }
    if (L.type == FL_LIGHT_POINT || L.type == FL_LIGHT_SPOT) {
        // PointIlluminant / SpotIlluminant::sample_li (point.cpp:12-19, spot.cpp:22-29): a delta
        // light (pdf 1), radiance color * intensity [* Falloff(-wi)] / evaluate_decay_rate, which
        // is always |d|^2 (illuminant.cpp:16-35 falls through its switch)
        const v3 pos = mk(L.cx, L.cy, L.cz);
        ls.wi = normalize(sub(pos, ref.p));
        ls.pdf = 1.f;
        ls.vis_kind = 1;
        ls.target = pos;
        const float dL = len(sub(pos, ref.p));
        const float strength = dL * dL;
        float li = L.radiance;
        if (L.type == FL_LIGHT_SPOT) {
            // SpotIlluminant::Falloff (spot.cpp:43-57)
            const float cosTheta = dot(normalize(neg(ls.wi)), normalize(mk(L.dx, L.dy, L.dz)));
            float fo;
            if (cosTheta < L.cos_cone) fo = 0.f;
            else if (cosTheta > L.cos_penumbra) fo = 1.f;
            else {
                const float t = clampr((cosTheta - L.cos_cone) / (L.cos_penumbra - L.cos_cone), 0.f, 1.f);
                fo = t * t * (3.f - 2.f * t);
            }
            li = li * fo;
        }
        ls.radiance = li / strength;
        return ls;
    }
    if (L.type == FL_LIGHT_DIRECTIONAL) {
        // DirectionalIlluminant::sample_li (directional.cpp:14-21): towards the light, the
        // visibility target 2 * worldRadius (1000) away
        ls.wi = mk(L.dx, L.dy, L.dz);
        ls.pdf = 1.f;
        ls.vis_kind = 1;
        ls.target = add(ref.p, mul(ls.wi, 2.f * 1000.f));
        ls.radiance = L.radiance;
        return ls;
    }
    const float z = 1.f - 2.f * ux;
    const float rr = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float phi = 2.f * kPi * uy;
    ls.wi = mk(rr * fl_cos(phi), rr * fl_sin(phi), z);
    ls.pdf = kInv4Pi;
    ls.vis_kind = 2;
    ls.radiance = L.radiance;
    return ls;
}

__device__ inline bool light_is_delta(const LightDev &L) {
    return L.type == FL_LIGHT_POINT || L.type == FL_LIGHT_SPOT || L.type == FL_LIGHT_DIRECTIONAL;
}

// Illuminant::pdf_li
static __device__ __noinline__ float light_pdf_li(const LightDev &L, const float *__restrict__ soup, const Hit &ref, v3 wi) {
    if (L.type == FL_LIGHT_TRIANGLE) {
        const v3 o = spawn_origin(ref.p, ref.n, wi);
        v3 p, n;
        if (!tri_intersect_ref(tri_v(soup, L.tri, 0), tri_v(soup, L.tri, 1), tri_v(soup, L.tri, 2), o, wi,
                               kShadowEpsilon, __int_as_float(0x7f800000), p, n))
            return 0.f;
        float pdf = len2(sub(ref.p, p)) / (absdot(n, neg(wi)) * L.area);
        if (isinf(pdf)) pdf = 0.f;
        return pdf;
    }
    if (L.type == FL_LIGHT_SPHERE) {
        const v3 o = spawn_origin(ref.p, ref.n, wi);
        const float t = sphere_hit(L, o, wi, kShadowEpsilon, __int_as_float(0x7f800000));
        if (t <= 0.f) return 0.f;
        const v3 p = add(o, mul(wi, t));
        const v3 nrm = normalize(sub(p, mk(L.cx, L.cy, L.cz)));
        const float cosl = dot(nrm, neg(wi));
        if (cosl <= 0.f) return 0.f;
        float pdf = len2(sub(ref.p, p)) / (cosl * L.area);
        if (isinf(pdf)) pdf = 0.f;
        return pdf;
    }
    if (L.type == FL_LIGHT_POINT || L.type == FL_LIGHT_SPOT || L.type == FL_LIGHT_DIRECTIONAL) return 0.f;
    return kInv4Pi;
}

__device__ inline float power_heuristic(float fPdf, float gPdf) {
    const float f = 1 * fPdf, g = 1 * gPdf;
    return (f * f) / (f * f + g * g);
}

}  // namespace fl
