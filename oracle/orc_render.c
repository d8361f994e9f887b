/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of the reference's path integrator with its BSDFs and lights, one
 * camera sample at a time, in the reference's operation order:
 *   PathIntegrator::Li            src/filianore/integrators/pathintegrator.cpp:12-87
 *   uniform_sample_all_lights     src/filianore/integrators/integrator.cpp:10-23
 *   estimate_direct               src/filianore/integrators/integrator.cpp:25-110
 *   power_heuristic               src/filianore/sampling/sampling.cpp:18-23
 *   BSDF evaluate/sample/pdf      src/filianore/shading/bsdf.cpp:6-151
 *   LambertBRDF                   src/filianore/shading/bxdfs/lambert.cpp:6-25
 *   concentric disk / cosine      src/filianore/core/shadingcore.h:65-89
 *   GGX D / Lambda / VNDF         src/filianore/shading/microfacets/ggx.cpp:12-57
 *   G, pdf                        src/filianore/shading/microfacets/microfacet.cpp:6-17
 *   MicrofacetReflectionBRDF      src/filianore/shading/bxdfs/microfacetreflection.cpp:13-61
 *   MicrofacetTransmissionBRDF    src/filianore/shading/closures/microfacettransmission.cpp:70-239
 *   FresnelSpecularBXDF           src/filianore/shading/closures/fresnelspecular.cpp:18-53
 *   FresnelDielectric/Conductor   src/filianore/shading/fresnel/fresneldielectric.cpp:8-38,
 *                                 src/filianore/shading/fresnel/fresnelconductor.cpp:9-33
 *   DiffuseAreaIlluminant         src/filianore/illuminants/diffusearea.cpp:12-39
 *   Shape::sample / Shape::pdf    src/filianore/shapes/shape.cpp:13-41
 *   Triangle::intersect / sample  src/filianore/shapes/triangle.cpp:13-154
 *   VisibilityEvaluator           src/filianore/illuminants/illuminant.cpp:40-50
 *   PhysicalCamera                src/filianore/cameras/physical.h:11-43, physical.cpp:4-22
 * The BVH hit record follows BVH::intersect (src/filianore/bvh/bvh.cpp:49-84) with the
 * primitive and shading normal filled in (its pError is gamma<int>(5) == 0).
 *
 * Features the reference lacks (environment light, analytic sphere light, hero
 * wavelengths, the render loop and its PCG32 seeding) are this project's own
 * definitions, shared with the GPU backend.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>

#define NL_MAX ORC_MAXLAMBDA
#define INF_F (__builtin_inff())

enum {
    BSDF_REFLECTION = 1 << 0,
    BSDF_TRANSMISSION = 1 << 1,
    BSDF_DIFFUSE = 1 << 2,
    BSDF_GLOSSY = 1 << 3,
    BSDF_SPECULAR = 1 << 4,
    BSDF_ALL = 31
};

typedef struct { float c[NL_MAX]; } spec;

typedef struct {
    const fl_scene_desc *sc;
    const orc_tables *tab;
    orc_bvh *bvh;
    int32_t *tri_light;  /* light index per triangle or -1 */
    int mode, nl;
    spec *mat_refl60;    /* per material, 60-bin reflectance (BINS60 mode) */
    int has_env;
    float env_radiance;
    int emissive_tris;
    int corrected;       /* FL_RENDER_CORRECTED_GGX */
} scene_ctx;

/* ---------------------------------------------------------------- spectra */
static inline void sp_set(spec *s, int nl, float v) { for (int i = 0; i < nl; ++i) s->c[i] = v; }
static inline int sp_black(const spec *s, int nl) {
    for (int i = 0; i < nl; ++i) if (s->c[i] != 0.f) return 0;
    return 1;
}
static inline float sp_max(const spec *s, int nl) {
    float m = s->c[0];
    for (int i = 1; i < nl; ++i) m = m > s->c[i] ? m : s->c[i];
    return m;
}

/* ---------------------------------------------------------------- rays / hits */
typedef struct { v3 o, d; float tmin, tmax; } ray3;

typedef struct {
    float t;
    v3 p, pError, wo, n, ns;
    int32_t prim;   /* triangle id, or -2 - light index for a sphere-light hit */
    float b1, b2;   /* barycentrics of the triangle's second and third vertex */
} isect_t;

static float sphere_hit(const fl_light *L, const ray3 *r) {
    /* analytic sphere: smallest root in (tmin, tmax), geometric form */
    v3 c = v3m(L->center[0], L->center[1], L->center[2]);
    v3 oc = v3_sub(r->o, c);
    float a = v3_dot(r->d, r->d);
    float b = v3_dot(oc, r->d);
    float cc = v3_dot(oc, oc) - L->radius * L->radius;
    float disc = b * b - a * cc;
    if (disc < 0.f || a == 0.f) return -1.f;
    float sq = sqrtf(disc);
    float t0 = (-b - sq) / a, t1 = (-b + sq) / a;
    if (t0 > r->tmin && t0 < r->tmax) return t0;
    if (t1 > r->tmin && t1 < r->tmax) return t1;
    return -1.f;
}

/* Scene::intersect -> BVH::intersect, plus analytic sphere lights */
static int scene_intersect(const scene_ctx *S, const ray3 *r, isect_t *is, uint64_t *rays) {
    float ot[4] = {r->o.x, r->o.y, r->o.z, r->tmin};
    float dt[4] = {r->d.x, r->d.y, r->d.z, r->tmax};
    orc_ray rr;
    orc_ray_precompute(ot, dt, &rr);
    float t, u, v;
    int32_t id = orc_bvh_closest(S->bvh, &rr, &t, &u, &v, NULL, NULL);
    ++*rays;
    float best = id >= 0 ? t : r->tmax;
    int32_t sphere = -1;
    for (uint32_t l = 0; l < S->sc->n_lights; ++l) {
        const fl_light *L = &S->sc->lights[l];
        if (L->type != FL_LIGHT_SPHERE) continue;
        ray3 r2 = *r;
        r2.tmax = best;
        float ts = sphere_hit(L, &r2);
        if (ts > 0.f && ts < best) { best = ts; sphere = (int32_t)l; }
    }
    if (id < 0 && sphere < 0) return 0;
    is->t = best;
    is->p = v3_add(r->o, v3_mul(r->d, best));
    is->pError = v3m(0.f, 0.f, 0.f);
    is->wo = v3_norm(v3_neg(r->d));
    if (sphere >= 0) {
        const fl_light *L = &S->sc->lights[sphere];
        is->n = v3_norm(v3_sub(is->p, v3m(L->center[0], L->center[1], L->center[2])));
        is->prim = -2 - sphere;
    } else {
        const float *tv = S->sc->verts + 9 * (size_t)id;
        v3 v0 = v3m(tv[0], tv[1], tv[2]), v1 = v3m(tv[3], tv[4], tv[5]), v2 = v3m(tv[6], tv[7], tv[8]);
        is->n = v3_norm(v3_cross(v3_sub(v1, v0), v3_sub(v2, v0)));
        is->prim = id;
    }
    is->b1 = sphere >= 0 ? 0.f : u;
    is->b2 = sphere >= 0 ? 0.f : v;
    is->ns = is->n;
    return 1;
}

/* The hit's texture coordinates uv0 (1 - b1 - b2) + uv1 b1 + uv2 b2 in this order; (0, 0)
 * without uvs, as BVH::intersect (bvh/bvh.cpp:69-71) leaves them */
static void hit_uv(const scene_ctx *S, const isect_t *is, float *u, float *v) {
    *u = *v = 0.f;
    if (!S->sc->uvs || is->prim < 0) return;
    const float *t = S->sc->uvs + 6 * (size_t)is->prim;
    float w = 1.f - is->b1 - is->b2;
    *u = t[0] * w + t[2] * is->b1 + t[4] * is->b2;
    *v = t[1] * w + t[3] * is->b1 + t[5] * is->b2;
}

/* ImageMapTexture::evaluate (shading/textures/imagemap.cpp:36-62): the nearest texel's RGB;
 * for j past the last row the reference sets i = height - 1 and reads outside the image,
 * here j is clamped too */
static void image_texel(const fl_image *im, float u, float v, float rgb[3]) {
    int i = (int)(u * (float)im->width);
    int j = (int)((1.f - v) * (float)im->height - 0.001f);
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > im->width - 1) i = im->width - 1;
    if (j > im->height - 1) { i = im->height - 1; j = im->height - 1; }
    if (i > im->width - 1) i = im->width - 1;
    const uint8_t *px = im->rgb + 3 * (size_t)i + 3 * (size_t)im->width * (size_t)j;
    for (int k = 0; k < 3; ++k) rgb[k] = (float)(int)px[k] / 255.f;
}

static int32_t prim_light(const scene_ctx *S, int32_t prim) {
    if (prim >= 0) return S->tri_light[prim];
    if (prim <= -2) return -2 - prim;
    return -1;
}

/* ---------------------------------------------------------------- shading frame */
typedef struct {
    v3 ng, ns, s, t;
    int type;        /* FL_MAT_* */
    float eta;       /* BSDF::eta */
    spec R;          /* reflectance */
    float ax, ay;    /* GGX alphas */
    float mat_eta, mat_k;
    int nl;
    int corrected;   /* FL_RENDER_CORRECTED_GGX */
    /* StandardSurfaceMaterial (FL_MAT_STANDARD): the lobes in the order
     * compute_scattering_functions adds them and their parameters */
    int std_n, std_lobes[5];
    spec kd, ks, kt, sheen, coat;
    spec metal_eta, metal_k;         /* measured metal (lobe 9) */
    float tf_ior, tf_thickness;      /* thin film (lobe 10) over a medium of IOR mat_eta */
    float wl[NL_MAX];                /* the path's wavelengths (bin starts in the 60-bin mode) */
    float kd_weight, on_A, on_B;     /* OrenNayarBRDF(kd, kdweight, 90 * kdrough) */
    float fb_A, fb_B;                /* the blended lobe's OrenNayarBRDF(kd, kdweight, kdrough) */
    float ks_weight, ro;
    int fresnel_type;
    float sheen_weight, sheen_rough;
    float coat_weight, coat_ior, coat_gloss;
} bsdf_t;

static v3 to_local(const bsdf_t *b, v3 v) { return v3m(v3_dot(v, b->s), v3_dot(v, b->t), v3_dot(v, b->ns)); }
static v3 to_world(const bsdf_t *b, v3 v) {
    return v3_add(v3_add(v3_mul(b->s, v.x), v3_mul(b->t, v.y)), v3_mul(b->ns, v.z));
}

static inline float cos2t(v3 w) { return w.z * w.z; }
static inline float sin2t(v3 w) { float v = 1.f - cos2t(w); return v > 0.f ? v : 0.f; }
static inline float sint(v3 w) { return sqrtf(sin2t(w)); }
static inline float tant(v3 w) { return sint(w) / w.z; }
static inline float tan2t(v3 w) { return sin2t(w) / cos2t(w); }
static inline float clampf_ref(float v, float lo, float hi) { if (v < lo) return lo; return v > hi ? hi : v; }
static inline float cosphi(v3 w) { float st = sint(w); return st == 0.f ? 1.f : clampf_ref(w.x / st, -1.f, 1.f); }
static inline float sinphi(v3 w) { float st = sint(w); return st == 0.f ? 0.f : clampf_ref(w.y / st, -1.f, 1.f); }
static inline float cos2phi(v3 w) { return cosphi(w) * cosphi(w); }
static inline float sin2phi(v3 w) { return sinphi(w) * sinphi(w); }
static inline int same_hemi(v3 a, v3 b) { return a.z * b.z > 0; }

/* ---- GGX (ggx.cpp) */
static float ggx_D(const bsdf_t *b, v3 wh) {
    float tan2Theta = tan2t(wh);
    if (isinf(tan2Theta)) return 0.f;
    const float cos4Theta = cos2t(wh) * cos2t(wh);
    float e = (cos2phi(wh) / (b->ax * b->ax) + sin2phi(wh) / (b->ay * b->ay)) * tan2Theta;
    return 1.f / (ORC_PI * b->ax * b->ay * cos4Theta * (1 + e) * (1 + e));
}
static float ggx_lambda(const bsdf_t *b, v3 w) {
    float absTanTheta = fabsf(tant(w));
    if (isinf(absTanTheta)) return 0.f;
    float alpha = sqrtf(cos2phi(w) * b->ax * b->ax + sin2phi(w) * b->ay * b->ay);
    float a2t2 = (alpha * absTanTheta) * (alpha * absTanTheta);
    return (-1 + sqrtf(1.f + a2t2)) / 2;
}
static float ggx_G(const bsdf_t *b, v3 wo, v3 wi) { return 1 / (1 + ggx_lambda(b, wo) + ggx_lambda(b, wi)); }
/* MicrofacetDistribution::pdf (microfacet.cpp:14-16): D |cos theta_h| (quirk Q1); the
 * corrected mode uses the visible-normal density G1(wo) |wo.wh| D(wh) / |cos theta_o| */
static float ggx_pdf(const bsdf_t *b, v3 wo, v3 wh) {
    if (b->corrected) {
        if (wo.z == 0.f) return 0.f;
        return ggx_D(b, wh) * fabsf(v3_dot(wo, wh)) / ((1.f + ggx_lambda(b, wo)) * fabsf(wo.z));
    }
    return ggx_D(b, wh) * fabsf(wh.z);
}
static v3 ggx_sample_wh_upper(const bsdf_t *b, v3 wo, float ux, float uy);
/* GGXDistribution::sample_wh (ggx.cpp:32-57) samples the upper hemisphere even for
 * wo.z < 0 (quirk Q2); the corrected mode samples around -wo and flips back */
static v3 ggx_sample_wh(const bsdf_t *b, v3 wo, float ux, float uy) {
    if (b->corrected && wo.z < 0.f) return v3_neg(ggx_sample_wh_upper(b, v3_neg(wo), ux, uy));
    return ggx_sample_wh_upper(b, wo, ux, uy);
}
static v3 ggx_sample_wh_upper(const bsdf_t *b, v3 wo, float ux, float uy) {
    v3 vh = v3_norm(v3m(wo.x * b->ax, wo.y * b->ay, wo.z));
    if (vh.z < 0) vh = v3_neg(vh);
    float lensq = vh.x * vh.x + vh.y * vh.y;
    v3 T1 = lensq > 0 ? v3_div(v3m(-vh.y, vh.x, 0.f), sqrtf(lensq)) : v3m(1.f, 0.f, 0.f);
    v3 T2 = v3_cross(vh, T1);
    float r = sqrtf(ux);
    float phi = 2.f * ORC_PI * uy;
    float t1 = r * cosf(phi);
    float t2 = r * sinf(phi);
    float s = (float)((1.f + vh.z) * 0.5);
    t2 = (1.f - s) * sqrtf(1 - (t1 * t1)) + (s * t2);
    float zz = 1.f - t1 * t1 - t2 * t2;
    v3 Nh = v3_add(v3_add(v3_mul(T1, t1), v3_mul(T2, t2)), v3_mul(vh, sqrtf(zz > 0.f ? zz : 0.f)));
    return v3_norm(v3m(b->ax * Nh.x, b->ay * Nh.y, Nh.z > 1e-6f ? Nh.z : 1e-6f));
}

/* ---- Fresnel (fresneldielectric.cpp:8-38 with local copies, fresnelconductor.cpp:9-33) */
static float fr_dielectric(float cosThetaI, float etaI, float etaT) {
    cosThetaI = clampf_ref(cosThetaI, -1.f, 1.f);
    int enter = cosThetaI > 0.0;
    if (!enter) { float tmp = etaI; etaI = etaT; etaT = tmp; cosThetaI = fabsf(cosThetaI); }
    float m = 1.f - cosThetaI * cosThetaI;
    float sinThetaI = sqrtf(m > 0.f ? m : 0.f);
    float sinThetaT = etaI / etaT * sinThetaI;
    if (sinThetaT >= 1) return 1.f;
    float m2 = 1 - sinThetaT * sinThetaT;
    float cosThetaT = sqrtf(m2 > 0.f ? m2 : 0.f);
    float Rparl = (etaT * cosThetaI - etaI * cosThetaT) / (etaT * cosThetaI + etaI * cosThetaT);
    float Rperp = (etaI * cosThetaI - etaT * cosThetaT) / (etaI * cosThetaI + etaT * cosThetaT);
    return (float)((Rparl * Rparl + Rperp * Rperp) * 0.5);
}
static float fr_conductor(float cosI, float etaT_, float k_) {
    /* constant eta/k over wavelength: every spectral sample is the same */
    cosI = fabsf(cosI);
    cosI = clampf_ref(cosI, -1.f, 1.f);
    float eta = etaT_ / 1.f;
    float etak = k_ / 1.f;
    float cosThetaI2 = cosI * cosI;
    float sinThetaI2 = (float)(1. - cosThetaI2);
    float eta2 = eta * eta;
    float etak2 = etak * etak;
    float t0 = eta2 - etak2 - sinThetaI2;
    float a2plusb2 = sqrtf(t0 * t0 + 4.f * eta2 * etak2);
    float t1 = a2plusb2 + cosThetaI2;
    float a = sqrtf(0.5f * (a2plusb2 + t0));
    float t2 = (float)2 * cosI * a;
    float Rs = (t1 - t2) / (t1 + t2);
    float t3 = cosThetaI2 * a2plusb2 + sinThetaI2 * sinThetaI2;
    float t4 = t2 * sinThetaI2;
    float Rp = Rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (Rp + Rs);
}

/* ---- lobes. Lobe ids: 0 lambert, 1 microfacet reflection, 2 microfacet transmission, 3 fresnel specular */
/* lobes: 0 Lambert, 1 GGX microfacet reflection, 2 GGX microfacet transmission,
 * 3 FresnelSpecular (R = T = the material colour), and the StandardSurface lobes
 * 4 Oren-Nayar, 5 Fresnel-blended diffuse + specular, 6 Estevez sheen, 7 GTR1 clear coat,
 * 8 FresnelSpecular with R = ks, T = kt, 9 GGX with the measured-metal conductor Fresnel,
 * 10 GGX with the thin-film Fresnel, 11 diffuse transmission */
static int lobe_type(int lobe) {
    switch (lobe) {
    case 0: return BSDF_REFLECTION | BSDF_DIFFUSE;
    case 1: return BSDF_REFLECTION | BSDF_GLOSSY;
    case 2: return BSDF_TRANSMISSION | BSDF_GLOSSY;
    case 4: return BSDF_REFLECTION | BSDF_DIFFUSE;
    case 5: case 6: case 7: case 9: case 10: return BSDF_REFLECTION | BSDF_GLOSSY;
    case 11: return BSDF_TRANSMISSION | BSDF_DIFFUSE;
    default: return BSDF_REFLECTION | BSDF_TRANSMISSION | BSDF_SPECULAR;
    }
}
static int bsdf_lobes(const bsdf_t *b, int *lobes) {
    switch (b->type) {
    case FL_MAT_LAMBERT: lobes[0] = 0; return 1;
    case FL_MAT_CONDUCTOR: lobes[0] = 1; return 1;
    case FL_MAT_ROUGH_DIELECTRIC: lobes[0] = 1; lobes[1] = 2; return 2;
    case FL_MAT_STANDARD:
        for (int i = 0; i < b->std_n; ++i) lobes[i] = b->std_lobes[i];
        return b->std_n;
    default: lobes[0] = 3; return 1;
    }
}

/* ---- StandardSurface lobes */
/* OrenNayarBRDF::OrenNayarBRDF (orennayar.cpp:6-12): sigma in degrees */
static void oren_nayar_ab(float sigma_deg, float *A, float *B) {
    float sigma = (ORC_PI / 180.f) * sigma_deg;
    float sigma2 = sigma * sigma;
    *A = 1.f - (sigma2 / (2.f * (sigma2 + 0.33f)));
    *B = 0.45f * sigma2 / (sigma2 + 0.09f);
}
/* OrenNayarBRDF::evaluate (orennayar.cpp:14-39) */
static void oren_nayar_eval(const spec *R, float weight, float A, float B, v3 wo, v3 wi, int nl, spec *out) {
    float sinThetaI = sint(wi), sinThetaO = sint(wo);
    float maxCos = 0.f;
    if (sinThetaI > 1e-4 && sinThetaO > 1e-4) {
        float sinPhiI = sinphi(wi), cosPhiI = cosphi(wi), sinPhiO = sinphi(wo), cosPhiO = cosphi(wo);
        float dCos = cosPhiI * cosPhiO + sinPhiI * sinPhiO;
        maxCos = dCos > 0.f ? dCos : 0.f;
    }
    float sinAlpha, tanBeta;
    if (fabsf(wi.z) > fabsf(wo.z)) { sinAlpha = sinThetaO; tanBeta = sinThetaI / fabsf(wi.z); }
    else { sinAlpha = sinThetaI; tanBeta = sinThetaO / fabsf(wo.z); }
    float v = (A + B * maxCos * sinAlpha * tanBeta);
    for (int i = 0; i < nl; ++i) out->c[i] = R->c[i] * ORC_INV_PI * v * weight;
}
/* cosine_hemisphere_sample (shadingcore.h:65-89), flipped to wo's side */
static v3 cos_hemi(v3 wo, float ux, float uy) {
    float ox = ux * 2.f - 1.f, oy = uy * 2.f - 1.f, dx, dy;
    if (ox == 0 && oy == 0) { dx = 0.f; dy = 0.f; }
    else {
        float theta, r;
        if (fabsf(ox) > fabsf(oy)) { r = ox; theta = ORC_PI_OVER_4 * (oy / ox); }
        else { r = oy; theta = ORC_PI_OVER_2 - ORC_PI_OVER_4 * (ox / oy); }
        dx = r * cosf(theta); dy = r * sinf(theta);
    }
    float zz = 1.f - dx * dx - dy * dy;
    v3 w = v3m(dx, dy, sqrtf(zz > 0.f ? zz : 0.f));
    if (wo.z < 0) w.z *= -1.f;
    return w;
}
static v3 reflect_wh(v3 wo, v3 wh) { return v3_sub(v3_mul(v3_mul(wh, 2.f), v3_dot(wo, wh)), wo); }
/* EstevezSheenDistribution (estevez.cpp:8-34) */
static float est_D(float r, v3 wh) {
    float inv = 1.f / r;
    return (2.f + inv) * powf(sint(wh), inv) / (2.f * ORC_PI);
}
static float est_plerp(float r, float p0, float p1) { return ((1.f - r) * (1.f - r)) * p0 + (1.f - ((1.f - r) * (1.f - r))) * p1; }
static float est_lambda(float r, v3 w) {
    float a = est_plerp(r, 25.3245f, 21.5473f), b = est_plerp(r, 3.32435f, 3.82987f), c = est_plerp(r, 0.16801f, 0.19823f);
    float d = est_plerp(r, -1.27393f, -1.97760f), e = est_plerp(r, -4.85967f, -4.32054f);
#define EST_L(v) (a / (1.f + b * powf((v), c)) + (d * (v)) + e)
    float ac = fabsf(w.z);
    if (ac < 0.5f) return expf(EST_L(ac));
    float ex = 2.f * EST_L(0.5f) - EST_L(1.f - ac);
#undef EST_L
    return expf(ex);
}
/* ClearcoatReflectionBRDF helpers (clearcoat.cpp:6-19) */
static float gtr1(float cosTheta, float alpha) {
    float alpha2 = alpha * alpha;
    return (alpha2 - 1) / (ORC_PI * logf(alpha2) * (1 + (alpha2 - 1) * cosTheta * cosTheta));
}
/* smithG_GGX calls the unqualified sqrt, which resolves to the double-precision C function:
 * the sum and the division are carried in double and rounded to float on return */
static float smith_g_ggx(float cosTheta, float alpha) {
    float alpha2 = alpha * alpha, cosTheta2 = cosTheta * cosTheta;
    return (float)(1.f / (cosTheta + sqrt((double)(alpha2 + cosTheta2 - alpha2 * cosTheta2))));
}
static int matches(int type, int flags) { return (type & flags) == type; }

/* ThinFilmInteference::evaluate (fresnel/thinfilm.cpp:8-58) with extIOR 1 and the amplitude
 * coefficients of fresnel/fresnel.h:9-23, at the path's wavelengths. The reference's
 * sin^2 ratios divide a quotient by itself, so both equal 1 - cos^2 (kept). */
static void thin_film_fresnel(const bsdf_t *b, float cosThetaI, spec *F) {
    const float extIOR = 1.f, tfIOR = b->tf_ior, mIOR = b->mat_eta, thickness = b->tf_thickness;
    float sinSqrd1 = ((extIOR / tfIOR) / (extIOR / tfIOR)) * (1 - cosThetaI * cosThetaI);
    float sinSqrd2 = ((extIOR / mIOR) / (extIOR / mIOR)) * (1 - cosThetaI * cosThetaI);
    if ((sinSqrd1 > 1) || (sinSqrd2 > 1)) { sp_set(F, b->nl, 1.f); return; }
    float cos1 = sqrtf(1 - sinSqrd1);
    float cos2 = sqrtf(1 - sinSqrd2);
#define SP_R(n1, n2, ci, ct) (((n1) * (ci) - (n2) * (ct)) / ((n1) * (ci) + (n2) * (ct)))
#define SP_T(n1, n2, ci, ct) ((2.f * (n1) * (ci)) / ((n1) * (ci) + (n2) * (ct)))
#define PP_R(n1, n2, ci, ct) (((n2) * (ci) - (n1) * (ct)) / ((n1) * (ct) + (n2) * (ci)))
#define PP_T(n1, n2, ci, ct) ((2.f * (n1) * (ci)) / ((n1) * (ct) + (n2) * (ci)))
    float alphaSP = SP_R(tfIOR, extIOR, cos1, cosThetaI) * SP_R(mIOR, tfIOR, cos1, cos2);
    float alphaPP = PP_R(tfIOR, extIOR, cos1, cosThetaI) * PP_R(mIOR, tfIOR, cos1, cos2);
    float betaSP = SP_T(extIOR, tfIOR, cosThetaI, cos1) * SP_T(tfIOR, mIOR, cos1, cos2);
    float betaPP = PP_T(extIOR, tfIOR, cosThetaI, cos1) * PP_T(tfIOR, mIOR, cos1, cos2);
#undef SP_R
#undef SP_T
#undef PP_R
#undef PP_T
    float delta10 = tfIOR < extIOR ? ORC_PI : 0.f;
    float delta12 = tfIOR < mIOR ? ORC_PI : 0.f;
    float delta = delta10 + delta12;
    float beamRatio = (mIOR * cos2) / (extIOR * cosThetaI);
    for (int i = 0; i < b->nl; ++i) {
        float wavelength = b->wl[i];
        float phi = (2.f * ORC_PI / wavelength) * (2.f * tfIOR * thickness * cos1) + delta;
        float cp = cosf(phi);
        float ts = (betaSP * betaSP) / ((alphaSP * alphaSP) - (2.f * alphaSP * cp) + 1.f);
        float tp = (betaPP * betaPP) / ((alphaPP * alphaPP) - (2.f * alphaPP * cp) + 1.f);
        F->c[i] = 1.f - (ts + tp) * 0.5f * beamRatio;
    }
}

/* lobe evaluate (spectrum) */
static void lobe_eval(const bsdf_t *b, int lobe, v3 wo, v3 wi, spec *out) {
    int nl = b->nl;
    if (lobe == 0) {
        for (int i = 0; i < nl; ++i) out->c[i] = b->R.c[i] * ORC_INV_PI * 1.f;
        return;
    }
    if (lobe == 1) {
        float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = v3_add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { sp_set(out, nl, 0.f); return; }
        wh = v3_norm(wh);
        v3 whf = v3_dot(wh, v3m(0.f, 0.f, 1.f)) < 0.f ? v3_neg(wh) : wh;
        float cF = v3_dot(wi, whf);
        float F = b->type == FL_MAT_CONDUCTOR ? fr_conductor(cF, b->mat_eta, b->mat_k) : fr_dielectric(cF, 1.f, b->mat_eta);
        float D = ggx_D(b, wh), G = ggx_G(b, wo, wi);
        float den = 4.f * cosThetaO * cosThetaI;
        for (int i = 0; i < nl; ++i) out->c[i] = b->R.c[i] * 1.f * D * G * F / den;
        return;
    }
    if (lobe == 2) {
        if (same_hemi(wo, wi)) { sp_set(out, nl, 0.f); return; }
        float cosThetaO = wo.z, cosThetaI = wi.z;
        if (cosThetaI == 0 || cosThetaO == 0) { sp_set(out, nl, 0.f); return; }
        float eta = wo.z > 0 ? (b->mat_eta / 1.f) : (1.f / b->mat_eta);
        v3 wh = v3_norm(v3_add(wo, v3_mul(wi, eta)));
        if (wh.z < 0) wh = v3_neg(wh);
        if (v3_dot(wo, wh) * v3_dot(wi, wh) > 0) { sp_set(out, nl, 0.f); return; }
        float F = fr_dielectric(v3_dot(wo, wh), 1.f, b->mat_eta);
        float sqrtDenom = v3_dot(wo, wh) + eta * v3_dot(wi, wh);
        float factor = (1 / eta);
        float v = fabsf(ggx_D(b, wh) * ggx_G(b, wo, wi) * eta * eta * v3_absdot(wi, wh) * v3_absdot(wo, wh) * factor * factor /
                        (cosThetaI * cosThetaO * sqrtDenom * sqrtDenom));
        for (int i = 0; i < nl; ++i) out->c[i] = (1.f - F) * b->R.c[i] * v;
        return;
    }
    if (lobe == 4) { oren_nayar_eval(&b->kd, b->kd_weight, b->on_A, b->on_B, wo, wi, nl, out); return; }
    if (lobe == 5) {
        /* FresnelBlendedDiffuseSpecularBRDF::evaluate (fresnelblendeddiffspec.cpp:18-38) */
        float r1 = 1.f - .5f * fabsf(wi.z);
        float r1pow5 = (r1 * r1) * (r1 * r1) * r1;
        float r2 = 1.f - .5f * fabsf(wo.z);
        float r2pow5 = (r2 * r2) * (r2 * r2) * r2;
        spec on;
        oren_nayar_eval(&b->kd, b->kd_weight, b->fb_A, b->fb_B, wo, wi, nl, &on);
        v3 wh = v3_add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) { sp_set(out, nl, 0.f); return; }
        wh = v3_norm(wh);
        float cF = v3_dot(wi, wh);
        float D = ggx_D(b, wh);
        float den = (4.f * v3_absdot(wi, wh) * fmaxf(fabsf(wi.z), fabsf(wo.z)));
        float R1 = 1.f - cF;
        for (int i = 0; i < nl; ++i) {
            float diffuse = (28.f / 23.f) * on.c[i] * (1.f - b->ro) * (1 - r1pow5) * (1 - r2pow5);
            float F;
            if (b->fresnel_type == FL_FRESNEL_METALLIC) {
                /* SchlickMetallic::evaluate (schlickmetallic.cpp:7-10), r0 = ks */
                F = b->ks.c[i] + (1.f - b->ks.c[i]) * (R1 * R1 * R1 * R1 * R1);
            } else {
                /* SchlickDielectric::evaluate (schlickdielectric.cpp:7-11) */
                F = b->ro + ((R1 * R1) * (R1 * R1) * R1) * (1.f - b->ro);
            }
            float specular = D * F / den;
            specular = b->ks.c[i] * specular * b->ks_weight;
            out->c[i] = diffuse + specular;
        }
        return;
    }
    if (lobe == 6) {
        /* MicrofacetReflectionBRDF::evaluate (microfacetreflection.cpp:11-28) with the Estevez
         * distribution and FresnelNull */
        float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = v3_add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { sp_set(out, nl, 0.f); return; }
        wh = v3_norm(wh);
        float D = est_D(b->sheen_rough, wh);
        float G = 1.f / (1.f + est_lambda(b->sheen_rough, wo) + est_lambda(b->sheen_rough, wi));
        float den = 4.f * cosThetaO * cosThetaI;
        for (int i = 0; i < nl; ++i) out->c[i] = b->sheen.c[i] * b->sheen_weight * D * G * 1.f / den;
        return;
    }
    if (lobe == 9 || lobe == 10) {
        /* MicrofacetReflectionBRDF::evaluate (microfacetreflection.cpp:13-32) with R = 1 and the
         * measured-metal FresnelConductor (weight ks_weight) or the thin film (weight 1) */
        float cosThetaO = fabsf(wo.z), cosThetaI = fabsf(wi.z);
        v3 wh = v3_add(wi, wo);
        if (cosThetaI == 0 || cosThetaO == 0 || (wh.x == 0 && wh.y == 0 && wh.z == 0)) { sp_set(out, nl, 0.f); return; }
        wh = v3_norm(wh);
        v3 whf = v3_dot(wh, v3m(0.f, 0.f, 1.f)) < 0.f ? v3_neg(wh) : wh;
        float cF = v3_dot(wi, whf);
        spec F;
        if (lobe == 9) for (int i = 0; i < nl; ++i) F.c[i] = fr_conductor(cF, b->metal_eta.c[i], b->metal_k.c[i]);
        else thin_film_fresnel(b, cF, &F);
        float weight = lobe == 9 ? b->ks_weight : 1.f;
        float D = ggx_D(b, wh), G = ggx_G(b, wo, wi);
        float den = 4.f * cosThetaO * cosThetaI;
        for (int i = 0; i < nl; ++i) out->c[i] = 1.f * weight * D * G * F.c[i] / den;
        return;
    }
    if (lobe == 11) { oren_nayar_eval(&b->kd, b->kd_weight, b->on_A, b->on_B, wo, wi, nl, out); return; }
    if (lobe == 7) {
        /* ClearcoatReflectionBRDF::evaluate (clearcoat.cpp:28-41) */
        v3 wh = v3_add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) { sp_set(out, nl, 0.f); return; }
        wh = v3_norm(wh);
        float Dr = gtr1(fabsf(wh.z), b->coat_gloss);
        float Fr = fr_dielectric(v3_dot(wo, wh), 1.f, b->coat_ior);
        float Gr = smith_g_ggx(fabsf(wo.z), .25f) * smith_g_ggx(fabsf(wi.z), .25f);
        for (int i = 0; i < nl; ++i) out->c[i] = b->coat.c[i] * Fr * b->coat_weight * Gr * Dr / 4;
        return;
    }
    sp_set(out, nl, 0.f);
}

static float lobe_pdf(const bsdf_t *b, int lobe, v3 wo, v3 wi) {
    if (lobe == 0) return same_hemi(wo, wi) ? fabsf(wi.z) * ORC_INV_PI : 0.f;
    if (lobe == 1) {
        if (!same_hemi(wo, wi)) return 0.f;
        v3 wh = v3_norm(v3_add(wo, wi));
        return ggx_pdf(b, wo, wh) / (4.f * v3_dot(wo, wh));
    }
    if (lobe == 2) {
        if (same_hemi(wo, wi)) return 0.f;
        float eta = wo.z > 0 ? (b->mat_eta / 1.f) : (1.f / b->mat_eta);
        v3 wh = v3_norm(v3_add(wo, v3_mul(wi, eta)));
        if (v3_dot(wo, wh) * v3_dot(wi, wh) > 0) return 0.f;
        float sqrtDenom = v3_dot(wo, wh) + eta * v3_dot(wi, wh);
        float dwh_dwi = fabsf((eta * eta * v3_dot(wi, wh)) / (sqrtDenom * sqrtDenom));
        return ggx_pdf(b, wo, wh) * dwh_dwi;
    }
    if (lobe == 4) return same_hemi(wo, wi) ? fabsf(wi.z) * ORC_INV_PI : 0.f;
    if (lobe == 5) {
        /* fresnelblendeddiffspec.cpp:61-67 */
        if (!same_hemi(wo, wi)) return 0;
        v3 wh = v3_norm(v3_add(wo, wi));
        float pdf_wh = ggx_pdf(b, wo, wh);
        return .5f * (fabsf(wi.z) * ORC_INV_PI + pdf_wh / (4 * v3_dot(wo, wh)));
    }
    if (lobe == 6) {
        /* MicrofacetReflectionBRDF::pdf with MicrofacetDistribution::pdf = D |cos theta_h| */
        if (!same_hemi(wo, wi)) return 0.f;
        v3 wh = v3_norm(v3_add(wo, wi));
        return est_D(b->sheen_rough, wh) * fabsf(wh.z) / (4.f * v3_dot(wo, wh));
    }
    if (lobe == 9 || lobe == 10) {
        if (!same_hemi(wo, wi)) return 0.f;
        v3 wh = v3_norm(v3_add(wo, wi));
        return ggx_pdf(b, wo, wh) / (4.f * v3_dot(wo, wh));
    }
    /* DiffuseTransmission::pdf (bxdfs/diffusetransmission.cpp:29-31) */
    if (lobe == 11) return !same_hemi(wo, wi) ? fabsf(wi.z) * ORC_INV_PI : 0.f;
    if (lobe == 7) {
        /* clearcoat.cpp:70-80 */
        if (!same_hemi(wo, wi)) return 0;
        v3 wh = v3_add(wi, wo);
        if (wh.x == 0 && wh.y == 0 && wh.z == 0) return 0;
        wh = v3_norm(wh);
        float Dr = gtr1(fabsf(wh.z), b->coat_gloss);
        return Dr * fabsf(wh.z) / (4 * v3_dot(wo, wh));
    }
    return 0.f;
}

/* lobe sample; *type may be overwritten by the lobe (fresnel specular) */
static void lobe_sample(const bsdf_t *b, int lobe, v3 wo, v3 *wi, float ux, float uy, float *pdf, int *type, spec *f) {
    int nl = b->nl;
    if (lobe == 0) {
        /* concentric_sample_disk + cosine_hemisphere_sample, shadingcore.h:65-89 */
        float ox = ux * 2.f - 1.f, oy = uy * 2.f - 1.f;
        float dx, dy;
        if (ox == 0 && oy == 0) { dx = 0.f; dy = 0.f; }
        else {
            float theta, r;
            if (fabsf(ox) > fabsf(oy)) { r = ox; theta = ORC_PI_OVER_4 * (oy / ox); }
            else { r = oy; theta = ORC_PI_OVER_2 - ORC_PI_OVER_4 * (ox / oy); }
            dx = r * cosf(theta); dy = r * sinf(theta);
        }
        float zz = 1.f - dx * dx - dy * dy;
        *wi = v3m(dx, dy, sqrtf(zz > 0.f ? zz : 0.f));
        if (wo.z < 0) wi->z *= -1.f;
        *pdf = lobe_pdf(b, 0, wo, *wi);
        lobe_eval(b, 0, wo, *wi, f);
        return;
    }
    if (lobe == 1) {
        if (wo.z == 0) { sp_set(f, nl, 0.f); return; }
        v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (v3_dot(wo, wh) < 0) { sp_set(f, nl, 0.f); return; }
        /* reflect(wo, wh) = wh*2*dot(wo,wh) - wo */
        *wi = v3_sub(v3_mul(v3_mul(wh, 2.f), v3_dot(wo, wh)), wo);
        if (!same_hemi(wo, *wi)) { sp_set(f, nl, 0.f); return; }
        *pdf = ggx_pdf(b, wo, wh) / (4.f * v3_dot(wo, wh));
        lobe_eval(b, 1, wo, *wi, f);
        return;
    }
    if (lobe == 2) {
        if (wo.z == 0) { sp_set(f, nl, 0.f); return; }
        v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (v3_dot(wo, wh) < 0) { sp_set(f, nl, 0.f); return; }
        float eta = wo.z > 0 ? (1.f / b->mat_eta) : (b->mat_eta / 1.f);
        /* refract, geometry.h:314-330 */
        float cosI = v3_dot(wo, wh);
        float m = 1.f - (cosI * cosI);
        float sinI2 = m > 0.f ? m : 0.f;
        float sinT2 = eta * eta * sinI2;
        if (sinT2 >= 1) { sp_set(f, nl, 0.f); return; }
        float cosT = sqrtf(1 - sinT2);
        *wi = v3_add(v3_mul(wo, -eta), v3_mul(wh, (eta * cosI - cosT)));
        *pdf = lobe_pdf(b, 2, wo, *wi);
        lobe_eval(b, 2, wo, *wi, f);
        return;
    }
    if (lobe == 4) {
        *wi = cos_hemi(wo, ux, uy);
        *pdf = lobe_pdf(b, 4, wo, *wi);
        lobe_eval(b, 4, wo, *wi, f);
        return;
    }
    if (lobe == 5) {
        /* fresnelblendeddiffspec.cpp:40-59 */
        if (ux < .5) {
            float u0 = 2 * ux;
            if (u0 > 1.f - ORC_SHADOW_EPSILON) u0 = 1.f - ORC_SHADOW_EPSILON;
            *wi = cos_hemi(wo, u0, uy);
        } else {
            float u0 = 2 * (ux - .5f);
            if (u0 > 1.f - ORC_SHADOW_EPSILON) u0 = 1.f - ORC_SHADOW_EPSILON;
            v3 wh = ggx_sample_wh(b, wo, u0, uy);
            *wi = reflect_wh(wo, wh);
            if (!same_hemi(wo, *wi)) { sp_set(f, nl, 0.f); return; }
        }
        *pdf = lobe_pdf(b, 5, wo, *wi);
        lobe_eval(b, 5, wo, *wi, f);
        return;
    }
    if (lobe == 6) {
        /* MicrofacetReflectionBRDF::sample (microfacetreflection.cpp:30-52); the Estevez
         * sample_wh draws a cosine-weighted normal on wo's side (estevez.cpp:36-42) */
        if (wo.z == 0) { sp_set(f, nl, 0.f); return; }
        v3 wh = cos_hemi(wo, ux, uy);
        if (v3_dot(wo, wh) < 0) { sp_set(f, nl, 0.f); return; }
        *wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, *wi)) { sp_set(f, nl, 0.f); return; }
        *pdf = est_D(b->sheen_rough, wh) * fabsf(wh.z) / (4.f * v3_dot(wo, wh));
        lobe_eval(b, 6, wo, *wi, f);
        return;
    }
    if (lobe == 9 || lobe == 10) {
        /* MicrofacetReflectionBRDF::sample (microfacetreflection.cpp:34-56) */
        if (wo.z == 0) { sp_set(f, nl, 0.f); return; }
        v3 wh = ggx_sample_wh(b, wo, ux, uy);
        if (v3_dot(wo, wh) < 0) { sp_set(f, nl, 0.f); return; }
        *wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, *wi)) { sp_set(f, nl, 0.f); return; }
        *pdf = ggx_pdf(b, wo, wh) / (4.f * v3_dot(wo, wh));
        lobe_eval(b, lobe, wo, *wi, f);
        return;
    }
    if (lobe == 11) {
        /* DiffuseTransmission::sample (bxdfs/diffusetransmission.cpp:16-27): a cosine-weighted
         * direction on the side away from wo */
        *wi = cos_hemi(v3m(0.f, 0.f, 1.f), ux, uy);
        if (wo.z > 0) wi->z *= -1.f;
        *pdf = lobe_pdf(b, 11, wo, *wi);
        lobe_eval(b, 11, wo, *wi, f);
        return;
    }
    if (lobe == 7) {
        /* clearcoat.cpp:43-68 */
        if (wo.z == 0) { sp_set(f, nl, 0.f); return; }
        float alpha2 = b->coat_gloss * b->coat_gloss;
        float cosTheta = sqrtf(fmaxf(0.f, (1 - powf(alpha2, 1 - ux)) / (1 - alpha2)));
        float sinTheta = sqrtf(fmaxf(0.f, 1 - cosTheta * cosTheta));
        float phi = 2 * ORC_PI * uy;
        v3 wh = v3m(sinTheta * cosf(phi), sinTheta * sinf(phi), cosTheta);
        if (!same_hemi(wo, wh)) wh = v3_neg(wh);
        *wi = reflect_wh(wo, wh);
        if (!same_hemi(wo, *wi)) { sp_set(f, nl, 0.f); return; }
        *pdf = lobe_pdf(b, 7, wo, *wi);
        lobe_eval(b, 7, wo, *wi, f);
        return;
    }
    /* fresnel specular (lobe 3; lobe 8 with R = ks, T = kt) */
    const spec *Rs = lobe == 8 ? &b->ks : &b->R;
    const spec *Ts = lobe == 8 ? &b->kt : &b->R;
    float F = fr_dielectric(wo.z, 1.f, b->mat_eta);
    if (ux < F) {
        *wi = v3m(-wo.x, -wo.y, wo.z);
        *type = BSDF_SPECULAR | BSDF_REFLECTION;
        *pdf = F;
        float ac = fabsf(wi->z);
        for (int i = 0; i < nl; ++i) f->c[i] = Rs->c[i] * F / ac;
    } else {
        int entering = wo.z > 0;
        float etaI = entering ? 1.f : b->mat_eta;
        float etaT = entering ? b->mat_eta : 1.f;
        v3 n = v3_dot(v3m(0.f, 0.f, 1.f), wo) < 0.f ? v3m(-0.f, -0.f, -1.f) : v3m(0.f, 0.f, 1.f);
        float eta = etaI / etaT;
        float cosI = v3_dot(wo, n);
        float m = 1.f - (cosI * cosI);
        float sinI2 = m > 0.f ? m : 0.f;
        float sinT2 = eta * eta * sinI2;
        if (sinT2 >= 1) { sp_set(f, nl, 0.f); return; }
        float cosT = sqrtf(1 - sinT2);
        *wi = v3_add(v3_mul(wo, -eta), v3_mul(n, (eta * cosI - cosT)));
        float sc = (etaI * etaI) / (etaT * etaT);
        *type = BSDF_SPECULAR | BSDF_TRANSMISSION;
        *pdf = 1.f - F;
        float ac = fabsf(wi->z);
        for (int i = 0; i < nl; ++i) {
            float ft = Ts->c[i] * (1.f - F);
            ft *= sc;
            f->c[i] = ft / ac;
        }
    }
}

static int bsdf_num_components(const bsdf_t *b, int flags) {
    int lobes[5], n = bsdf_lobes(b, lobes), c = 0;
    for (int i = 0; i < n; ++i) if (matches(lobe_type(lobes[i]), flags)) ++c;
    return c;
}

/* BSDF::evaluate, bsdf.cpp:30-50 */
static void bsdf_eval(const bsdf_t *b, v3 woW, v3 wiW, int flags, spec *out) {
    v3 wi = to_local(b, wiW), wo = to_local(b, woW);
    sp_set(out, b->nl, 0.f);
    if (wo.z == 0) return;
    int reflect = v3_dot(wiW, b->ng) * v3_dot(woW, b->ng) > 0;
    int lobes[5], n = bsdf_lobes(b, lobes);
    for (int i = 0; i < n; ++i) {
        int ty = lobe_type(lobes[i]);
        if (matches(ty, flags) && ((reflect && (ty & BSDF_REFLECTION)) || (!reflect && (ty & BSDF_TRANSMISSION)))) {
            spec f;
            lobe_eval(b, lobes[i], wo, wi, &f);
            for (int k = 0; k < b->nl; ++k) out->c[k] += f.c[k];
        }
    }
}

/* BSDF::pdf, bsdf.cpp:127-151 */
static float bsdf_pdf(const bsdf_t *b, v3 woW, v3 wiW, int flags) {
    int lobes[5], n = bsdf_lobes(b, lobes);
    if (n == 0) return 0.f;
    v3 wi = to_local(b, wiW), wo = to_local(b, woW);
    if (wo.z == 0) return 0.f;
    float pdf = 0.f;
    int mc = 0;
    for (int i = 0; i < n; ++i)
        if (matches(lobe_type(lobes[i]), flags)) { ++mc; pdf += lobe_pdf(b, lobes[i], wo, wi); }
    return mc > 0 ? pdf / (float)mc : 0.f;
}

/* BSDF::sample, bsdf.cpp:52-125. Returns 0 when *pdf was left untouched (wo.z == 0). */
static void bsdf_sample(const bsdf_t *b, v3 woW, v3 *wiW, float ux, float uy, float *pdf, int flags, int *sampledType,
                        spec *f) {
    int lobes[5], n = bsdf_lobes(b, lobes);
    int mc = 0;
    for (int i = 0; i < n; ++i) if (matches(lobe_type(lobes[i]), flags)) ++mc;
    sp_set(f, b->nl, 0.f);
    if (mc == 0) { *pdf = 0.f; *sampledType = 0; return; }
    int comp = (int)floorf(ux * mc);
    if (comp > mc - 1) comp = mc - 1;
    int chosen = -1, count = comp;
    for (int i = 0; i < n; ++i)
        if (matches(lobe_type(lobes[i]), flags) && count-- == 0) { chosen = lobes[i]; break; }
    float urx = ux * mc - comp;
    if (urx > 1.f - ORC_SHADOW_EPSILON) urx = 1.f - ORC_SHADOW_EPSILON;
    v3 wi = v3m(0.f, 0.f, 0.f), wo = to_local(b, woW);
    if (wo.z == 0) return;
    *pdf = 0.f;
    int ctype = lobe_type(chosen);
    *sampledType = ctype;
    lobe_sample(b, chosen, wo, &wi, urx, uy, pdf, sampledType, f);
    if (*pdf == 0) { *sampledType = 0; sp_set(f, b->nl, 0.f); return; }
    *wiW = to_world(b, wi);
    if (!(ctype & BSDF_SPECULAR) && mc > 1) {
        for (int i = 0; i < n; ++i)
            if (lobes[i] != chosen && matches(lobe_type(lobes[i]), flags)) *pdf += lobe_pdf(b, lobes[i], wo, wi);
    }
    if (mc > 1) *pdf /= mc;
    if (!(ctype & BSDF_SPECULAR)) {
        int reflect = v3_dot(*wiW, b->ng) * v3_dot(woW, b->ng) > 0;
        sp_set(f, b->nl, 0.f);
        for (int i = 0; i < n; ++i) {
            int ty = lobe_type(lobes[i]);
            if (matches(ty, flags) && ((reflect && (ty & BSDF_REFLECTION)) || (!reflect && (ty & BSDF_TRANSMISSION)))) {
                spec g;
                lobe_eval(b, lobes[i], wo, wi, &g);
                for (int k = 0; k < b->nl; ++k) f->c[k] += g.c[k];
            }
        }
    }
}

/* the texel rule for n uv pairs (tests) */
void orc_image_texels(const fl_image *im, const float *uv, uint32_t n, float *rgb) {
    for (uint32_t i = 0; i < n; ++i) image_texel(im, uv[2 * i], uv[2 * i + 1], rgb + 3 * (size_t)i);
}

/* Material::bump_evaluate (materials/material.cpp:8-31) with the bump map's red channel as
 * height: the shading normal of a triangle hit. dpdu, dpdv follow Triangle::intersect
 * (shapes/triangle.cpp:33-52) over the vertex uvs (all zero without uvs). */
static v3 bump_normal(const scene_ctx *S, const isect_t *is, const fl_image *im) {
    const float *tv = S->sc->verts + 9 * (size_t)is->prim;
    v3 p1 = v3m(tv[0], tv[1], tv[2]), p2 = v3m(tv[3], tv[4], tv[5]), p3 = v3m(tv[6], tv[7], tv[8]);
    float uv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (S->sc->uvs) memcpy(uv, S->sc->uvs + 6 * (size_t)is->prim, sizeof(uv));
    float duv02x = uv[0] - uv[4], duv02y = uv[1] - uv[5];
    float duv12x = uv[2] - uv[4], duv12y = uv[3] - uv[5];
    v3 dp02 = v3_sub(p1, p3), dp12 = v3_sub(p2, p3);
    float determinant = duv02x * duv12y - duv02y * duv12x;
    int degenerate = fabs((double)determinant) < 1e-8;
    v3 dpdu = v3m(0.f, 0.f, 0.f), dpdv = v3m(0.f, 0.f, 0.f);
    if (!degenerate) {
        float invDet = 1.f / determinant;
        dpdu = v3_mul(v3_sub(v3_mul(dp02, duv12y), v3_mul(dp12, duv02y)), invDet);
        dpdv = v3_mul(v3_add(v3_mul(dp02, -duv12x), v3_mul(dp12, duv02x)), invDet);
    }
    if (degenerate || v3_len2(v3_cross(dpdu, dpdv)) == 0.f)
        orc_coordinate_system(v3_cross(v3_sub(p2, p1), v3_sub(p3, p1)), &dpdu, &dpdv);
    float u, v, rgb[3];
    hit_uv(S, is, &u, &v);
    const float du = 0.0005f, dv = 0.0005f;
    image_texel(im, u + du, v, rgb);
    float uDisplace = rgb[0];
    image_texel(im, u, v + dv, rgb);
    float vDisplace = rgb[0];
    image_texel(im, u, v, rgb);
    float displace = rgb[0];
    v3 bu = v3_add(dpdu, v3_mul(v3_mul(is->n, (uDisplace - displace) / du), 4.f));
    v3 bv = v3_add(dpdv, v3_mul(v3_mul(is->n, (vDisplace - displace) / dv), 4.f));
    /* set_shading_geometry (core/interaction.cpp:20-33): the normal of (bu, bv) on n's side */
    v3 ns = v3_norm(v3_cross(bu, bv));
    return v3_dot(ns, is->n) < 0.f ? v3_neg(ns) : ns;
}

/* Material::compute_scattering_functions for the supported materials */
static void make_bsdf(const scene_ctx *S, const isect_t *is, const float *lambda, bsdf_t *b) {
    b->nl = S->nl;
    b->ng = is->n;
    b->ns = is->ns;
    orc_coordinate_system(b->ns, &b->s, &b->t);
    b->s = v3_norm(b->s);
    uint32_t mi = 0;
    if (is->prim >= 0 && S->sc->tri_material) mi = S->sc->tri_material[is->prim];
    const fl_material *m = &S->sc->materials[mi];
    b->type = m->type;
    b->mat_eta = m->eta;
    b->mat_k = m->k;
    float a = m->roughness * m->roughness;
    b->ax = a > 0.001f ? a : 0.001f;
    b->ay = b->ax;
    b->eta = (m->type == FL_MAT_ROUGH_DIELECTRIC || m->type == FL_MAT_SMOOTH_DIELECTRIC) ? m->eta : 1.f;
    b->corrected = S->corrected;
    if (m->type == FL_MAT_LAMBERT && m->texture > 0) {
        /* LambertMaterial with an ImageMapTexture (materials/lambert.cpp:8-15) */
        float u, v, rgb[3];
        hit_uv(S, is, &u, &v);
        image_texel(&S->sc->images[m->texture - 1], u, v, rgb);
        orc_reflectance(S->tab, rgb, S->mode, lambda, b->R.c);
    } else if (m->type == FL_MAT_LAMBERT) {
        if (S->mode == FL_SPECTRAL_BINS60) b->R = S->mat_refl60[mi];
        else orc_reflectance(S->tab, m->rgb, S->mode, lambda, b->R.c);
    } else {
        sp_set(&b->R, b->nl, 1.f);
    }
    if (m->type == FL_MAT_STANDARD) {
        /* StandardSurfaceMaterial::compute_scattering_functions (standardsurface.cpp:72-159)
         * with constant textures */
        const fl_standard_surface *p = &S->sc->standard_surfaces[m->standard];
        b->eta = (p->ks_weight > 0 && p->kt_weight > 0) ? p->ks_ior : 1.f;
        b->mat_eta = p->ks_ior;
        if (p->kd_texture > 0) {
            float u, v, rgb[3];
            hit_uv(S, is, &u, &v);
            image_texel(&S->sc->images[p->kd_texture - 1], u, v, rgb);
            orc_reflectance(S->tab, rgb, S->mode, lambda, b->kd.c);
        } else {
            orc_reflectance(S->tab, p->kd, S->mode, lambda, b->kd.c);
        }
        orc_reflectance(S->tab, p->ks, S->mode, lambda, b->ks.c);
        orc_reflectance(S->tab, p->kt, S->mode, lambda, b->kt.c);
        orc_reflectance(S->tab, p->sheen_color, S->mode, lambda, b->sheen.c);
        orc_reflectance(S->tab, p->coat_color, S->mode, lambda, b->coat.c);
        b->kd_weight = p->kd_weight;
        oren_nayar_ab(p->kd_roughness * 90.f, &b->on_A, &b->on_B);
        oren_nayar_ab(p->kd_roughness, &b->fb_A, &b->fb_B);  /* the blended lobe passes the raw roughness as sigma */
        float aspect = sqrtf(1.f - p->ks_anisotropic * 0.9f);
        float a2 = p->ks_roughness * p->ks_roughness;
        b->ax = fmaxf(.001f, a2 / aspect);
        b->ay = fmaxf(.001f, a2 * aspect);
        b->ro = ((1.f - p->ks_ior) / (1.f + p->ks_ior)) * ((1.f - p->ks_ior) / (1.f + p->ks_ior));
        b->ks_weight = p->ks_weight;
        b->fresnel_type = p->fresnel_type;
        b->sheen_weight = p->sheen_weight;
        b->sheen_rough = fmaxf(.001f, p->sheen_roughness);
        b->coat_weight = p->coat_weight;
        b->coat_ior = p->coat_ior;
        b->coat_gloss = (1.f - p->coat_gloss) * .1f + p->coat_gloss * .001f;  /* lerp(gloss, .1, .001) */
        const int measured = p->fresnel_type == FL_FRESNEL_MEASURED_METAL;
        const int metal = (p->metal_type >= 0 && p->metal_type <= 8) ? p->metal_type : 0;  /* default: gold */
        for (int i = 0; i < b->nl; ++i) {
            if (S->mode == FL_SPECTRAL_BINS60) {
                b->metal_eta.c[i] = S->tab->metal[metal][0][i];
                b->metal_k.c[i] = S->tab->metal[metal][1][i];
                b->wl[i] = (float)(400 + 5 * i);
            } else {
                /* hero wavelengths read the 5 nm bin they fall in, clamped to 400..700 nm */
                int bin = (int)floorf((lambda[i] - 400.f) / 5.f);
                bin = bin < 0 ? 0 : (bin > ORC_NBINS - 1 ? ORC_NBINS - 1 : bin);
                b->metal_eta.c[i] = S->tab->metal[metal][0][bin];
                b->metal_k.c[i] = S->tab->metal[metal][1][bin];
                b->wl[i] = lambda[i];
            }
        }
        if (p->bump_texture > 0 && is->prim >= 0) {
            b->ns = bump_normal(S, is, &S->sc->images[p->bump_texture - 1]);
            orc_coordinate_system(b->ns, &b->s, &b->t);
            b->s = v3_norm(b->s);
        }
        b->tf_ior = p->thin_film_ior;
        b->tf_thickness = p->thin_film_thickness;
        b->std_n = 0;
        if ((p->kd_weight > 0 && p->ks_weight <= 0) || (p->kd_weight > 0 && p->ks_weight > 0 && measured))
            b->std_lobes[b->std_n++] = p->thin_walled ? 11 : 4;
        if (p->ks_weight > 0) b->std_lobes[b->std_n++] = p->kt_weight > 0 ? 8 : (measured ? 9 : 5);
        if (p->thin_film_thickness > 0) b->std_lobes[b->std_n++] = 10;
        if (p->sheen_weight > 0) b->std_lobes[b->std_n++] = 6;
        if (p->coat_weight > 0) b->std_lobes[b->std_n++] = 7;
    }
}

/* ---------------------------------------------------------------- lights */
/* Triangle::intersect (triangle.cpp:13-124): only p and n are used by Shape::pdf */
static int tri_intersect_ref(const float *tv, const ray3 *r, v3 *p, v3 *n) {
    v3 v1 = v3m(tv[0], tv[1], tv[2]), v2 = v3m(tv[3], tv[4], tv[5]), v3v = v3m(tv[6], tv[7], tv[8]);
    v3 e1 = v3_sub(v2, v1), e2 = v3_sub(v3v, v1);
    v3 nn = v3_cross(e1, e2);
    float det = -v3_dot(r->d, nn);
    v3 ao = v3_sub(r->o, v1);
    v3 dao = v3_cross(ao, r->d);
    float invDet = 1.f / det;
    float alpha = v3_dot(e2, dao) * invDet;
    float beta = -v3_dot(e1, dao) * invDet;
    float t = v3_dot(ao, nn) * invDet;
    if ((t < r->tmax && t > r->tmin) && alpha > 0 && beta > 0 && (alpha + beta) < 1.f) {
        if (v3_len2(nn) == 0) return 0;
        *p = v3_add(r->o, v3_mul(r->d, t));
        *n = v3_norm(v3_cross(v3_sub(v1, v3v), v3_sub(v2, v3v)));
        return 1;
    }
    return 0;
}

static float tri_area(const float *tv) {
    v3 v1 = v3m(tv[0], tv[1], tv[2]), v2 = v3m(tv[3], tv[4], tv[5]), v3v = v3m(tv[6], tv[7], tv[8]);
    return 0.5f * v3_len(v3_cross(v3_sub(v2, v1), v3_sub(v3v, v1)));
}

typedef struct {
    int kind;         /* 0 none, 1 finite point (segment test), 2 direction to infinity */
    v3 target;        /* light point (kind 1) */
} vis_t;

/* Illuminant::sample_li. Returns the radiance (constant over wavelength) via *Li. */
static int light_is_delta(const fl_light *L) {
    return L->type == FL_LIGHT_POINT || L->type == FL_LIGHT_SPOT || L->type == FL_LIGHT_DIRECTIONAL;
}

static float light_sample_li(const scene_ctx *S, int li, const isect_t *ref, float ux, float uy, v3 *wi, float *pdf,
                             vis_t *vis) {
    const fl_light *L = &S->sc->lights[li];
    vis->kind = 0;
    if (L->type == FL_LIGHT_TRIANGLE) {
        const float *tv = S->sc->verts + 9 * (size_t)L->tri;
        v3 p0 = v3m(tv[0], tv[1], tv[2]), p1 = v3m(tv[3], tv[4], tv[5]), p2 = v3m(tv[6], tv[7], tv[8]);
        /* Triangle::sample(u, pdf) */
        float uu = sqrtf(ux);
        float u1 = 1.f - uu;
        float u2 = uy * uu;
        v3 ip = v3_add(v3_add(v3_mul(p0, u1), v3_mul(p1, u2)), v3_mul(p2, (1.f - u1 - u2)));
        v3 in = v3_norm(v3_cross(v3_sub(p1, p0), v3_sub(p2, p0)));
        *pdf = 1.f / tri_area(tv);
        /* Shape::sample(isect, u, pdf) */
        v3 w = v3_sub(ip, ref->p);
        if (v3_len2(w) == 0) *pdf = 0.f;
        else {
            w = v3_norm(w);
            *pdf *= v3_len2(v3_sub(ref->p, ip)) / v3_absdot(in, v3_neg(w));
            if (isinf(*pdf)) *pdf = 0.f;
        }
        /* DiffuseAreaIlluminant::sample_li */
        if (*pdf == 0 || v3_len2(v3_sub(ip, ref->p)) == 0) { *pdf = 0.f; return 0.f; }
        *wi = v3_norm(v3_sub(ip, ref->p));
        vis->kind = 1;
        vis->target = ip;
        return v3_dot(in, v3m(-wi->x, -wi->y, -wi->z)) > 0.f ? L->radiance : 0.f;
    }
    if (L->type == FL_LIGHT_SPHERE) {
        /* uniform area sampling of the sphere, converted to solid angle */
        v3 c = v3m(L->center[0], L->center[1], L->center[2]);
        float z = 1.f - 2.f * ux;
        float rr = sqrtf(fmaxf(0.f, 1.f - z * z));
        float phi = 2.f * ORC_PI * uy;
        v3 nrm = v3m(rr * cosf(phi), rr * sinf(phi), z);
        v3 ip = v3_add(c, v3_mul(nrm, L->radius));
        float area = 4.f * ORC_PI * L->radius * L->radius;
        v3 w = v3_sub(ip, ref->p);
        float d2 = v3_len2(w);
        if (d2 == 0) { *pdf = 0.f; return 0.f; }
        w = v3_norm(w);
        float cosl = v3_dot(nrm, v3_neg(w));
        if (cosl <= 0.f) { *pdf = 0.f; return 0.f; }
        *pdf = d2 / (cosl * area);
        if (isinf(*pdf)) { *pdf = 0.f; return 0.f; }
        *wi = w;
        vis->kind = 1;
        vis->target = ip;
        return L->radiance;
    }
    if (L->type == FL_LIGHT_POINT || L->type == FL_LIGHT_SPOT) {
        /* PointIlluminant / SpotIlluminant::sample_li (point.cpp:12-19, spot.cpp:22-29);
         * evaluate_decay_rate falls through its switch to |d|^2 (illuminant.cpp:16-35) */
        v3 pos = v3m(L->center[0], L->center[1], L->center[2]);
        *wi = v3_norm(v3_sub(pos, ref->p));
        *pdf = 1.f;
        vis->kind = 1;
        vis->target = pos;
        float dL = v3_len(v3_sub(pos, ref->p));
        float strength = dL * dL;
        float li = L->radiance;
        if (L->type == FL_LIGHT_SPOT) {
            /* SpotIlluminant::Falloff (spot.cpp:43-57) */
            float cosCone = cosf(L->cone_angle), cosPen = cosf(L->penumbra_angle);
            float cosTheta = v3_dot(v3_norm(v3_neg(*wi)), v3_norm(v3m(L->direction[0], L->direction[1], L->direction[2])));
            float fo;
            if (cosTheta < cosCone) fo = 0.f;
            else if (cosTheta > cosPen) fo = 1.f;
            else {
                float t = clampf_ref((cosTheta - cosCone) / (cosPen - cosCone), 0.f, 1.f);
                fo = t * t * (3.f - 2.f * t);
            }
            li = li * fo;
        }
        return li / strength;
    }
    if (L->type == FL_LIGHT_DIRECTIONAL) {
        /* DirectionalIlluminant (directional.cpp:6-21): towards the light, target 2 * 1000 away */
        *wi = v3_norm(v3_neg(v3m(L->direction[0], L->direction[1], L->direction[2])));
        *pdf = 1.f;
        vis->kind = 1;
        vis->target = v3_add(ref->p, v3_mul(*wi, 2.f * 1000.f));
        return L->radiance;
    }
    /* environment: uniform sphere directions */
    float z = 1.f - 2.f * ux;
    float rr = sqrtf(fmaxf(0.f, 1.f - z * z));
    float phi = 2.f * ORC_PI * uy;
    *wi = v3m(rr * cosf(phi), rr * sinf(phi), z);
    *pdf = ORC_INV_4_PI;
    vis->kind = 2;
    return L->radiance;
}

/* Illuminant::pdf_li */
static float light_pdf_li(const scene_ctx *S, int li, const isect_t *ref, v3 wi) {
    const fl_light *L = &S->sc->lights[li];
    if (L->type == FL_LIGHT_TRIANGLE) {
        const float *tv = S->sc->verts + 9 * (size_t)L->tri;
        ray3 r = {orc_offset_point_origin(ref->p, ref->pError, ref->n, wi), wi, ORC_SHADOW_EPSILON, INF_F};
        v3 p, n;
        if (!tri_intersect_ref(tv, &r, &p, &n)) return 0.f;
        float pdf = v3_len2(v3_sub(ref->p, p)) / (v3_absdot(n, v3_neg(wi)) * tri_area(tv));
        if (isinf(pdf)) pdf = 0.f;
        return pdf;
    }
    if (L->type == FL_LIGHT_SPHERE) {
        ray3 r = {orc_offset_point_origin(ref->p, ref->pError, ref->n, wi), wi, ORC_SHADOW_EPSILON, INF_F};
        float t = sphere_hit(L, &r);
        if (t <= 0.f) return 0.f;
        v3 p = v3_add(r.o, v3_mul(r.d, t));
        v3 c = v3m(L->center[0], L->center[1], L->center[2]);
        v3 nrm = v3_norm(v3_sub(p, c));
        float area = 4.f * ORC_PI * L->radius * L->radius;
        float cosl = v3_dot(nrm, v3_neg(wi));
        if (cosl <= 0.f) return 0.f;
        float pdf = v3_len2(v3_sub(ref->p, p)) / (cosl * area);
        if (isinf(pdf)) pdf = 0.f;
        return pdf;
    }
    if (light_is_delta(L)) return 0.f;
    return ORC_INV_4_PI;
}

/* radiance leaving a hit on light li towards w (AreaIlluminant::L, diffusearea.cpp:37-39) */
static float light_L(const scene_ctx *S, int li, const isect_t *is, v3 w) {
    const fl_light *L = &S->sc->lights[li];
    if (L->type == FL_LIGHT_ENV) return 0.f;
    return v3_dot(is->n, w) > 0.f ? L->radiance : 0.f;
}

/* VisibilityEvaluator::unoccluded (illuminant.cpp:40-50): no hit, or the closest hit
 * carries an area light. Analytic sphere lights never occlude. */
static int unoccluded(const scene_ctx *S, const isect_t *p0, const vis_t *vis, v3 wi, uint64_t *rays) {
    ray3 r;
    if (vis->kind == 1) {
        v3 d = v3_sub(vis->target, p0->p);
        r.o = orc_offset_point_origin(p0->p, p0->pError, p0->n, d);
        r.d = d;
        r.tmin = ORC_SHADOW_EPSILON;
        r.tmax = 1.f - ORC_SHADOW_EPSILON;
    } else {
        r.o = orc_offset_point_origin(p0->p, p0->pError, p0->n, wi);
        r.d = wi;
        r.tmin = ORC_SHADOW_EPSILON;
        r.tmax = INF_F;
    }
    float ot[4] = {r.o.x, r.o.y, r.o.z, r.tmin};
    float dt[4] = {r.d.x, r.d.y, r.d.z, r.tmax};
    orc_ray rr;
    orc_ray_precompute(ot, dt, &rr);
    float t, u, v;
    int32_t id = orc_bvh_closest(S->bvh, &rr, &t, &u, &v, NULL, NULL);
    ++*rays;
    if (id < 0) return 1;
    return S->tri_light[id] >= 0;
}

static float power_heuristic(float fPdf, float gPdf) {
    float f = 1 * fPdf, g = 1 * gPdf;
    return (f * f) / (f * f + g * g);
}

typedef struct { uint64_t rays, shadow_rays, bounces; } counters;

/* estimate_direct, integrator.cpp:25-110 (area / sphere / environment lights are never delta) */
static void estimate_direct(const scene_ctx *S, const isect_t *it, const bsdf_t *b, float usx, float usy, int li,
                            float ulx, float uly, spec *Ld, counters *cn) {
    const int nl = S->nl;
    const int bsdfFlags = BSDF_ALL & ~BSDF_SPECULAR;
    sp_set(Ld, nl, 0.f);
    v3 wi = v3m(0.f, 0.f, 0.f);
    float illumPdf = 0, scatteringPdf = 0;
    vis_t vis;
    float Lrad = light_sample_li(S, li, it, ulx, uly, &wi, &illumPdf, &vis);
    if (illumPdf > 0 && Lrad != 0.f) {
        spec f;
        bsdf_eval(b, it->wo, wi, bsdfFlags, &f);
        float ad = v3_absdot(wi, it->ns);
        for (int i = 0; i < nl; ++i) f.c[i] *= ad;
        scatteringPdf = bsdf_pdf(b, it->wo, wi, bsdfFlags);
        if (!sp_black(&f, nl)) {
            ++cn->shadow_rays;
            if (!unoccluded(S, it, &vis, wi, &cn->rays)) Lrad = 0.f;
            if (Lrad != 0.f) {
                /* delta lights are not weighted (integrator.cpp:57-58) */
                float weight = light_is_delta(&S->sc->lights[li]) ? 1.f : power_heuristic(illumPdf, scatteringPdf);
                for (int i = 0; i < nl; ++i) Ld->c[i] += f.c[i] * Lrad * weight / illumPdf;
            }
        }
    }
    /* MIS - BSDF, not for delta lights (integrator.cpp:66) */
    if (!light_is_delta(&S->sc->lights[li])) {
        spec f;
        int sampledType = 0;
        bsdf_sample(b, it->wo, &wi, usx, usy, &scatteringPdf, bsdfFlags, &sampledType, &f);
        float ad = v3_absdot(wi, it->ns);
        for (int i = 0; i < nl; ++i) f.c[i] *= ad;
        int sampledSpecular = (sampledType & BSDF_SPECULAR) != 0;
        if (!sp_black(&f, nl) && scatteringPdf > 0) {
            float weight = 1.f;
            if (!sampledSpecular) {
                illumPdf = light_pdf_li(S, li, it, wi);
                if (illumPdf == 0) return;
                weight = power_heuristic(scatteringPdf, illumPdf);
            }
            ray3 r = {orc_offset_point_origin(it->p, it->pError, it->n, wi), wi, ORC_SHADOW_EPSILON, INF_F};
            isect_t li_is;
            float Lv = 0.f;
            if (scene_intersect(S, &r, &li_is, &cn->rays)) {
                if (prim_light(S, li_is.prim) == li) Lv = light_L(S, li, &li_is, v3_neg(wi));
            } else {
                const fl_light *L = &S->sc->lights[li];
                Lv = L->type == FL_LIGHT_ENV ? L->radiance : 0.f;
            }
            if (Lv != 0.f)
                for (int i = 0; i < nl; ++i) Ld->c[i] += f.c[i] * Lv * 1.f * weight / scatteringPdf;
        }
    }
}

/* PathIntegrator::Li, pathintegrator.cpp:12-87 */
static void path_Li(const scene_ctx *S, const fl_render_params *P, v3 o, v3 d, float tmin, float tmax,
                    const float *lambda, orc_pcg32 *rng, spec *L, counters *cn) {
    const int nl = S->nl;
    spec beta;
    sp_set(L, nl, 0.f);
    sp_set(&beta, nl, 1.f);
    ray3 ray = {o, d, tmin, tmax};
    int specularBounce = 0;
    float etaScale = 1.f;
    /* RenderParams (core/renderparams.h:5-10): diffuse, reflection, transmission depth */
    int depth[3] = {P->max_depth, P->max_depth, P->max_depth};
    if (P->flags & FL_RENDER_LOBE_DEPTHS) {
        depth[0] = P->diffuse_depth;
        depth[1] = P->reflection_depth;
        depth[2] = P->transmission_depth;
    }
    const float rrThreshold = P->rr_threshold;
    for (int bounces = 0;; ++bounces) {
        isect_t is;
        int hit = scene_intersect(S, &ray, &is, &cn->rays);
        if (bounces == 0 || specularBounce) {
            if (hit) {
                int li = prim_light(S, is.prim);
                if (li >= 0) {
                    float le = light_L(S, li, &is, v3_neg(ray.d));
                    for (int i = 0; i < nl; ++i) L->c[i] += beta.c[i] * le;
                }
            } else if (S->has_env) {
                /* escaped rays see the environment (Illuminant::le for infinite lights) */
                for (int i = 0; i < nl; ++i) L->c[i] += beta.c[i] * S->env_radiance;
            }
        }
        if (!hit) break;
        ++cn->bounces;
        bsdf_t b;
        make_bsdf(S, &is, lambda, &b);
        is.ns = b.ns;  /* a bump map changed the shading normal (isect->Shading.n) */
        if (bsdf_num_components(&b, BSDF_ALL & ~BSDF_SPECULAR) > 0) {
            spec Ls;
            sp_set(&Ls, nl, 0.f);
            for (uint32_t li = 0; li < S->sc->n_lights; ++li) {
                float ulx = orc_pcg32_nextf(rng), uly = orc_pcg32_nextf(rng);
                float usx = orc_pcg32_nextf(rng), usy = orc_pcg32_nextf(rng);
                spec e;
                estimate_direct(S, &is, &b, usx, usy, (int)li, ulx, uly, &e, cn);
                for (int i = 0; i < nl; ++i) Ls.c[i] += e.c[i];
            }
            for (int i = 0; i < nl; ++i) L->c[i] += beta.c[i] * Ls.c[i];
        }
        v3 wo = v3_neg(ray.d), wi = v3m(0.f, 0.f, 0.f);
        float pdf = 0.f;
        int flags = 0;
        spec f;
        float ux = orc_pcg32_nextf(rng), uy = orc_pcg32_nextf(rng);
        bsdf_sample(&b, wo, &wi, ux, uy, &pdf, BSDF_ALL, &flags, &f);
        if (sp_black(&f, nl) || pdf == 0) break;
        /* pathintegrator.cpp:55-65: the sampled lobe's own depth, tested with == */
        if (depth[0] == bounces && (flags & BSDF_DIFFUSE)) break;
        if ((depth[1] == bounces && (flags & BSDF_SPECULAR)) || (depth[1] == bounces && (flags & BSDF_GLOSSY))) break;
        if (depth[2] == bounces && (flags & BSDF_TRANSMISSION)) break;
        float ad = v3_absdot(wi, is.ns);
        for (int i = 0; i < nl; ++i) beta.c[i] *= f.c[i] * ad / pdf;
        specularBounce = (flags & BSDF_SPECULAR) != 0;
        if ((flags & BSDF_SPECULAR) && (flags & BSDF_TRANSMISSION)) {
            float eta = b.eta;
            etaScale *= (v3_dot(wo, is.n) > 0) ? (eta * eta) : 1.f / (eta * eta);
        }
        ray.o = orc_offset_point_origin(is.p, is.pError, is.n, wi);
        ray.d = wi;
        ray.tmin = ORC_SHADOW_EPSILON;
        ray.tmax = INF_F;
        spec rr;
        for (int i = 0; i < nl; ++i) rr.c[i] = beta.c[i] * etaScale;
        float mx = sp_max(&rr, nl);
        if (mx < rrThreshold && bounces > 3) {
            float q = 1.f - mx;
            if (q < 0.05f) q = 0.05f;
            if (orc_pcg32_nextf(rng) < q) break;
            for (int i = 0; i < nl; ++i) beta.c[i] /= 1.f - q;
        }
    }
}

/* ---------------------------------------------------------------- camera */
void orc_camera_init(const fl_camera *c, orc_camera *out) {
    v3 pos = v3m(c->position[0], c->position[1], c->position[2]);
    v3 at = v3m(c->look_at[0], c->look_at[1], c->look_at[2]);
    v3 up = v3m(c->up[0], c->up[1], c->up[2]);
    float focusDistance = v3_len(v3_sub(pos, at));
    float theta = c->vfov_deg * ORC_PI / 180.f;
    float halfHeight = tanf(theta / 2.f);
    float aspect = (float)c->width / (float)c->height;
    float halfWidth = aspect * halfHeight;
    v3 w = v3_norm(v3_sub(pos, at));
    /* flipCameraDirection = true: the orientation in which the camera looks at look_at */
    w = v3_mul(w, -1.f);
    v3 u = v3_norm(v3_cross(up, w));
    v3 v = v3_cross(w, u);
    w = v3_mul(w, -1.f);
    out->origin = pos;
    out->u = u;
    out->v = v;
    out->lower_left = v3_sub(v3_sub(v3_sub(pos, v3_mul(v3_mul(u, halfWidth), focusDistance)),
                                    v3_mul(v3_mul(v, focusDistance), halfHeight)),
                             v3_mul(w, focusDistance));
    out->horizontal = v3_mul(v3_mul(v3_mul(u, 2.f), halfWidth), focusDistance);
    out->vertical = v3_mul(v3_mul(v3_mul(v, 2.f), halfHeight), focusDistance);
    out->lens_radius = c->aperture / 2.f;  /* lensRadius = aperture / 2 (physical.h:20) */
}

/* The render loop the reference lacks: sample (s, t) of pixel p, PhysicalCamera::awaken_ray
 * with lens sample (0.5, 0.5) (a pinhole: the lens loop of physical.cpp:4-10 exits at once). */
void orc_camera_ray(const orc_camera *cam, const fl_camera *c, uint32_t pixel, orc_pcg32 *rng, v3 *o, v3 *d,
                    float *u_lambda) {
    float ux = orc_pcg32_nextf(rng), uy = orc_pcg32_nextf(rng);
    *u_lambda = orc_pcg32_nextf(rng);
    uint32_t px = pixel % (uint32_t)c->width, py = pixel / (uint32_t)c->width;
    float sx = ((float)px + ux) / (float)c->width;
    float sy = ((float)((uint32_t)c->height - 1u - py) + uy) / (float)c->height;
    v3 rd;
    if (cam->lens_radius > 0.f) {
        /* a lens: two more numbers, mapped with concentric_sample_disk (shadingcore.h:65-80)
         * in place of random_point_on_lens, whose rejection loop never draws a new sample */
        float lx = orc_pcg32_nextf(rng), ly = orc_pcg32_nextf(rng);
        float ox = lx * 2.f - 1.f, oy = ly * 2.f - 1.f, dx = 0.f, dy = 0.f;
        if (!(ox == 0 && oy == 0)) {
            float theta, r;
            if (fabsf(ox) > fabsf(oy)) { r = ox; theta = ORC_PI_OVER_4 * (oy / ox); }
            else { r = oy; theta = ORC_PI_OVER_2 - ORC_PI_OVER_4 * (ox / oy); }
            dx = cosf(theta) * r; dy = sinf(theta) * r;
        }
        rd = v3_mul(v3m(dx, dy, 0.f), cam->lens_radius);
    } else {
        /* random_point_on_lens((0.5, 0.5)) * lensRadius with lensRadius = 0 */
        v3 p = v3_sub(v3_mul(v3m(0.5f, 0.5f, 0.f), 2.f), v3m(1.f, 1.f, 0.f));
        rd = v3_mul(p, 0.f);
    }
    v3 offset = v3_add(v3_mul(cam->u, rd.x), v3_mul(cam->v, rd.y));
    *o = v3_add(cam->origin, offset);
    v3 dir = v3_sub(v3_sub(v3_add(v3_add(cam->lower_left, v3_mul(cam->horizontal, sx)), v3_mul(cam->vertical, sy)),
                           cam->origin),
                    offset);
    *d = v3_norm(dir);
}

/* hero wavelengths of lambda0: rotation by 85 nm, wrapped into [380, 720) */
static void hero_lambdas(float l0, float lambda[4]) {
    for (int j = 0; j < 4; ++j) {
        float l = l0 + 85.f * (float)j;
        lambda[j] = l >= 720.f ? l - 340.f : l;
    }
}

/* ---------------------------------------------------------------- driver */
typedef struct {
    const scene_ctx *S;
    const fl_camera *cam;
    const orc_camera *oc;
    const fl_render_params *P;
    const orc_render_opts *opts;
    double *film;
    uint32_t total;
    volatile uint32_t *next;
    counters cn;
    uint64_t paths;
} worker_arg;

static void *render_worker(void *argp) {
    worker_arg *a = (worker_arg *)argp;
    const scene_ctx *S = a->S;
    const int nl = S->nl;
    for (;;) {
        uint32_t start = __atomic_fetch_add(a->next, 64u, __ATOMIC_RELAXED);
        if (start >= a->total) break;
        uint32_t end = start + 64u < a->total ? start + 64u : a->total;
        for (uint32_t k = start; k < end; ++k) {
            uint32_t pixel = a->opts && a->opts->pixels ? a->opts->pixels[k] : k;
            double acc[3] = {0, 0, 0};
            for (int s = 0; s < a->P->spp; ++s) {
                orc_pcg32 rng;
                orc_pcg32_seed(&rng, pixel, 1u);
                uint64_t sidx = (uint64_t)a->P->sample_offset + (uint64_t)s;
                if (sidx) orc_pcg32_advance(&rng, (int64_t)(sidx << 16));
                v3 o, d;
                float ul;
                orc_camera_ray(a->oc, a->cam, pixel, &rng, &o, &d, &ul);
                float lambda[4];
                if (S->mode == FL_SPECTRAL_HERO4) hero_lambdas(380.f + ul * 340.f, lambda);
                spec L;
                path_Li(S, a->P, o, d, 0.f, INF_F, lambda, &rng, &L, &a->cn);
                double xyz[3];
                orc_xyz_from_spectrum(S->tab, S->mode, lambda, L.c, xyz);
                (void)nl;
                acc[0] += xyz[0]; acc[1] += xyz[1]; acc[2] += xyz[2];
                a->paths++;
            }
            a->film[3 * (size_t)pixel + 0] += acc[0];
            a->film[3 * (size_t)pixel + 1] += acc[1];
            a->film[3 * (size_t)pixel + 2] += acc[2];
        }
    }
    return NULL;
}

static void scene_ctx_init(scene_ctx *Sp, const fl_scene_desc *sc, const orc_tables *tab, const fl_render_params *P) {
    scene_ctx S;
    memset(&S, 0, sizeof(S));
    S.sc = sc;
    S.tab = tab;
    S.mode = P->spectral_mode;
    S.corrected = (P->flags & FL_RENDER_CORRECTED_GGX) != 0;
    S.nl = S.mode == FL_SPECTRAL_BINS60 ? ORC_NBINS : 4;
    S.bvh = orc_bvh_build(sc->verts, sc->n_tri);
    S.tri_light = (int32_t *)malloc(sizeof(int32_t) * (sc->n_tri ? sc->n_tri : 1));
    for (uint32_t i = 0; i < sc->n_tri; ++i) S.tri_light[i] = -1;
    for (uint32_t l = 0; l < sc->n_lights; ++l) {
        if (sc->lights[l].type == FL_LIGHT_TRIANGLE && sc->lights[l].tri < sc->n_tri) {
            S.tri_light[sc->lights[l].tri] = (int32_t)l;
            S.emissive_tris++;
        }
        if (sc->lights[l].type == FL_LIGHT_ENV) { S.has_env = 1; S.env_radiance = sc->lights[l].radiance; }
    }
    S.mat_refl60 = (spec *)malloc(sizeof(spec) * (sc->n_materials ? sc->n_materials : 1));
    for (uint32_t m = 0; m < sc->n_materials; ++m)
        orc_reflectance(tab, sc->materials[m].rgb, FL_SPECTRAL_BINS60, NULL, S.mat_refl60[m].c);
    *Sp = S;
}

static void scene_ctx_free(scene_ctx *S) {
    orc_bvh_free(S->bvh);
    free(S->tri_light);
    free(S->mat_refl60);
}

int orc_render(const fl_scene_desc *sc, const orc_tables *tab, const fl_camera *cam, const fl_render_params *P,
               const orc_render_opts *opts, double *film, orc_render_counts *counts) {
    if (!sc || !tab || !cam || !P || !film || cam->width <= 0 || cam->height <= 0 || P->spp <= 0) return -1;
    scene_ctx S;
    scene_ctx_init(&S, sc, tab, P);
    orc_camera oc;
    orc_camera_init(cam, &oc);
    uint32_t total = opts && opts->pixels ? opts->n_pixels : (uint32_t)cam->width * (uint32_t)cam->height;
    int nth = opts && opts->nthreads > 0 ? opts->nthreads : 1;
    if (nth > 256) nth = 256;
    volatile uint32_t next = 0;
    pthread_t th[256];
    worker_arg args[256];
    for (int k = 0; k < nth; ++k) {
        memset(&args[k], 0, sizeof(worker_arg));
        args[k].S = &S; args[k].cam = cam; args[k].oc = &oc; args[k].P = P; args[k].opts = opts;
        args[k].film = film; args[k].total = total; args[k].next = &next;
        pthread_create(&th[k], NULL, render_worker, &args[k]);
    }
    orc_render_counts c = {0, 0, 0, 0};
    for (int k = 0; k < nth; ++k) {
        pthread_join(th[k], NULL);
        c.paths += args[k].paths;
        c.rays += args[k].cn.rays;
        c.shadow_rays += args[k].cn.shadow_rays;
        c.bounces += args[k].cn.bounces;
    }
    if (counts) *counts = c;
    scene_ctx_free(&S);
    return 0;
}

/* The camera rays of sample `sample` of the given pixels, as the render loop makes them:
 * (o, tmin 0), (d, tmax inf), the generator state after the camera's draws and the hero
 * wavelength 380 + 340 u. */
void orc_camera_rays(const fl_camera *cam, const uint32_t *pixels, uint32_t n, uint32_t sample, float *org_tmin,
                     float *dir_tmax, uint64_t *rng_state, float *lambda0) {
    orc_camera oc;
    orc_camera_init(cam, &oc);
    for (uint32_t i = 0; i < n; ++i) {
        orc_pcg32 rng;
        orc_pcg32_seed(&rng, pixels[i], 1u);
        if (sample) orc_pcg32_advance(&rng, (int64_t)((uint64_t)sample << 16));
        v3 o, d;
        float ul;
        orc_camera_ray(&oc, cam, pixels[i], &rng, &o, &d, &ul);
        org_tmin[4 * i] = o.x; org_tmin[4 * i + 1] = o.y; org_tmin[4 * i + 2] = o.z; org_tmin[4 * i + 3] = 0.f;
        dir_tmax[4 * i] = d.x; dir_tmax[4 * i + 1] = d.y; dir_tmax[4 * i + 2] = d.z; dir_tmax[4 * i + 3] = INF_F;
        rng_state[i] = rng.state;
        lambda0[i] = 380.f + ul * 340.f;
    }
}

/* PathIntegrator::Li (pathintegrator.cpp:12-87) for n given rays: ray i starts from
 * generator state rng_state[i] (increment 3) and hero wavelength lambda0[i]; writes its
 * radiance (NL floats: 60 bins or 4 hero samples), the generator state after the path and
 * to_xyz of the radiance. The first ray's tmin and tmax are the given ones (Li copies
 * its ray argument). */
int orc_li(const fl_scene_desc *sc, const orc_tables *tab, const fl_render_params *P, uint32_t n,
           const float *org_tmin, const float *dir_tmax, const uint64_t *rng_state, const float *lambda0,
           float *radiance, uint64_t *rng_out, double *xyz) {
    if (!sc || !tab || !P) return -1;
    scene_ctx S;
    scene_ctx_init(&S, sc, tab, P);
    counters cn;
    memset(&cn, 0, sizeof(cn));
    for (uint32_t i = 0; i < n; ++i) {
        orc_pcg32 rng = {rng_state[i], 3u};
        float lambda[4] = {0.f, 0.f, 0.f, 0.f};
        if (S.mode == FL_SPECTRAL_HERO4) hero_lambdas(lambda0[i], lambda);
        spec L;
        v3 o = v3m(org_tmin[4 * i], org_tmin[4 * i + 1], org_tmin[4 * i + 2]);
        v3 d = v3m(dir_tmax[4 * i], dir_tmax[4 * i + 1], dir_tmax[4 * i + 2]);
        path_Li(&S, P, o, d, org_tmin[4 * i + 3], dir_tmax[4 * i + 3], lambda, &rng, &L, &cn);
        for (int k = 0; k < S.nl; ++k) radiance[(size_t)i * S.nl + k] = L.c[k];
        rng_out[i] = rng.state;
        orc_xyz_from_spectrum(S.tab, S.mode, lambda, L.c, xyz + 3 * (size_t)i);
    }
    scene_ctx_free(&S);
    return 0;
}

/* f(wo, wi) |cos theta_i| of a non-Lambert material (reflectance 1, so the same at every
 * wavelength) in its local frame (normal +z), for n directions wi: a reference-free check of
 * the estimators, whose expectation under constant light is this function's integral. */
void orc_bsdf_fcos(const fl_material *m, const float wo[3], uint32_t n, const float *wi, int corrected, float *out) {
    bsdf_t b;
    memset(&b, 0, sizeof(b));
    b.nl = 1;
    b.ng = b.ns = v3m(0.f, 0.f, 1.f);
    b.s = v3m(1.f, 0.f, 0.f);
    b.t = v3m(0.f, 1.f, 0.f);
    b.type = m->type;
    b.mat_eta = m->eta;
    b.mat_k = m->k;
    const float a = m->roughness * m->roughness;
    b.ax = b.ay = a > 0.001f ? a : 0.001f;
    b.eta = (m->type == FL_MAT_ROUGH_DIELECTRIC || m->type == FL_MAT_SMOOTH_DIELECTRIC) ? m->eta : 1.f;
    b.R.c[0] = 1.f;
    b.corrected = corrected;
    const v3 o = v3m(wo[0], wo[1], wo[2]);
    for (uint32_t i = 0; i < n; ++i) {
        const v3 d = v3m(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        spec f;
        bsdf_eval(&b, o, d, BSDF_ALL, &f);
        out[i] = f.c[0] * fabsf(d.z);
    }
}

