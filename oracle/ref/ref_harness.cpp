/*
 * Render driver for the reference's own integrator (test infrastructure only).
 *
 * filianore-core has no render loop, film or sampler with reproducible seeds (its
 * Whitenoise sampler seeds mt19937 from std::random_device,
 * src/filianore/sampling/samplers/whitenoise.h:25-28). This driver supplies them with the
 * same definitions the GPU backend uses, and otherwise runs the reference unchanged:
 *   - scene: one Triangle + Material + optional DiffuseAreaIlluminant per soup triangle
 *     (shapes/triangle.h, illuminants/diffusearea.h). Materials: LambertMaterial
 *     (shading/materials/lambert.h) with albedos upsampled by from_reflectance_rgb
 *     (color/spectrumoperations.cpp:113-147), and three compositions of the reference's
 *     BxDFs in the way StandardSurfaceMaterial builds them (materials/standardsurface.cpp:72-159):
 *     GGX conductor = MicrofacetReflectionBRDF(GGX(r^2), FresnelConductor(1, eta, k), 1, 1);
 *     rough dielectric = MicrofacetReflectionBRDF(GGX(r^2), FresnelDielectric(1, ior), 1, 1)
 *     + MicrofacetTransmissionBRDF(1, 1, 1, 1, 1, ior, GGX(r^2)) in a BSDF with eta = ior;
 *     smooth dielectric = FresnelSpecularBXDF(1, 1, 1, ior) in a BSDF with eta = ior;
 *   - camera: PhysicalCamera with aperture 0 and flipCameraDirection = true
 *     (cameras/physical.h:11-43): with the default false the camera faces away from
 *     its look-at point, with true it faces it;
 *   - integrator: PathIntegrator(RenderParams{spp, d, d, d}, rr) (integrators/pathintegrator.h);
 *   - sampler: a Sampler (sampling/sampler.h:10-19) over the vendored pcg32
 *     (src/ext/pcg32.h), seeded per (pixel, sample) with seed(pixel, 1) and advance(sample << 16);
 *     camera sample order: ux, uy, u_lambda (unused by the 60-bin spectra);
 *   - film: sums over samples of to_xyz(Li) in double (color/spectrumoperations.cpp:193-207).
 *
 * Usage:
 *   ref_render SCENE.bin OUT.bin     render a scene file written by tests/golden/scenefile.py
 *   ref_render SCENE.bin OUT.bin --forge   the same after InitializeForge (color/metallurgy.cpp:7-39),
 *                                    which nothing in the reference calls: without it the
 *                                    measured-metal spectra stay zero
 *   ref_render --tables OUT.bin      dump the raw and 60-bin spectral tables
 *   ref_render --metals OUT.bin      dump the measured metal curves (color/metallurgy.h) and the
 *                                    60-bin spectra InitializeForge makes of them
 *   ref_render --pcg OUT.bin         dump pcg32 known-answer sequences
 */
#include "filianore/cameras/physical.h"
#include "filianore/color/cie.h"
#include "filianore/color/metallurgy.h"
#include "filianore/color/spectruminits.h"
#include "filianore/color/spectrumoperations.h"
#include "filianore/core/interaction.h"
#include "filianore/core/primitive.h"
#include "filianore/core/scene.h"
#include "filianore/illuminants/diffusearea.h"
#include "filianore/illuminants/directional.h"
#include "filianore/illuminants/point.h"
#include "filianore/illuminants/spot.h"
#include "filianore/integrators/pathintegrator.h"
#include "filianore/sampling/sampler.h"
#include "filianore/shading/bsdf.h"
#include "filianore/shading/bxdfs/microfacetreflection.h"
#include "filianore/shading/closures/fresnelspecular.h"
#include "filianore/shading/closures/microfacettransmission.h"
#include "filianore/shading/fresnel/fresnelconductor.h"
#include "filianore/shading/fresnel/fresneldielectric.h"
#include "filianore/shading/materials/lambert.h"
#include "filianore/shading/materials/standardsurface.h"
#include "filianore/shading/microfacets/ggx.h"
#include "filianore/shading/textures/constant.h"
#include "filianore/shading/textures/imagemap.h"
#include "filianore/shapes/triangle.h"
#include "ext/pcg32.h"
#include "../../include/filianore_gpu.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace ref_shim {
extern std::vector<const filianore::Primitive *> g_primitives;
extern std::vector<float> g_uvs;
}

using namespace filianore;

namespace {

// The bump map's height: the red byte / 255 of the nearest texel, by ImageMapTexture's rule
// (shading/textures/imagemap.cpp:36-62). The reference has no float image texture.
class RedChannelTexture : public Texture<float> {
public:
    RedChannelTexture(int w, int h, std::vector<uint8_t> px) : w_(w), h_(h), px_(std::move(px)) {}
    float evaluate(const SurfaceInteraction &isect) const {
        int i = int(isect.uv.x * w_);
        int j = int((1.f - isect.uv.y) * h_ - 0.001f);
        if (i < 0) i = 0;
        if (j < 0) j = 0;
        if (i > w_ - 1) i = w_ - 1;
        if (j > h_ - 1) { i = h_ - 1; j = h_ - 1; }
        if (i > w_ - 1) i = w_ - 1;
        return int(px_[3 * i + 3 * w_ * j]) / 255.f;
    }

private:
    int w_, h_;
    std::vector<uint8_t> px_;
};

class PCG32Sampler : public Sampler {
public:
    void reset(uint64_t pixel, uint64_t sample) {
        rng.seed(pixel, 1u);
        if (sample) rng.advance((int64_t)(sample << 16));
    }
    float get_1d() override { return rng.nextFloat(); }
    Vector2f get_2d() override {
        float x = get_1d();
        float y = get_1d();
        return Vector2f(x, y);
    }
    void prepare_next_sample() override {}

private:
    pcg32 rng;
};

struct SceneFileHeader {
    char magic[8];
    uint32_t n_tri, n_mat, n_light, spp, max_depth, spectral_mode, sample_offset, nthreads, n_pixels;
    uint32_t diffuse_depth, reflection_depth, transmission_depth;  // RenderParams' three depths
    float rr_threshold;
    fl_camera cam;
};

template <typename T>
bool read_n(FILE *f, std::vector<T> &v, size_t n) {
    v.resize(n);
    return n == 0 || fread(v.data(), sizeof(T), n, f) == n;
}

// Materials composed from the reference's BxDF classes (see the header comment).
class ConductorMaterial : public Material {
public:
    ConductorMaterial(float alpha, float eta, float k) : alpha(alpha), eta(eta), k(k) {}
    void compute_scattering_functions(SurfaceInteraction *isect) const override {
        isect->bsdf = std::make_shared<BSDF>(*isect, 1.f);
        auto distribution = std::make_shared<GGXDistribution>(alpha, alpha);
        std::shared_ptr<Fresnel> fresnel =
            std::make_shared<FresnelConductor>(PrincipalSpectrum(1.f), PrincipalSpectrum(eta), PrincipalSpectrum(k));
        std::unique_ptr<BxDF> lobe =
            std::make_unique<MicrofacetReflectionBRDF>(distribution, fresnel, PrincipalSpectrum(1.f), 1.f);
        isect->bsdf->add(lobe);
    }

private:
    float alpha, eta, k;
};

class RoughDielectricMaterial : public Material {
public:
    RoughDielectricMaterial(float alpha, float ior) : alpha(alpha), ior(ior) {}
    void compute_scattering_functions(SurfaceInteraction *isect) const override {
        isect->bsdf = std::make_shared<BSDF>(*isect, ior);
        auto distribution = std::make_shared<GGXDistribution>(alpha, alpha);
        std::shared_ptr<Fresnel> fresnel = std::make_shared<FresnelDielectric>(1.f, ior);
        std::unique_ptr<BxDF> refl =
            std::make_unique<MicrofacetReflectionBRDF>(distribution, fresnel, PrincipalSpectrum(1.f), 1.f);
        isect->bsdf->add(refl);
        std::unique_ptr<BxDF> trans = std::make_unique<MicrofacetTransmissionBRDF>(
            PrincipalSpectrum(1.f), 1.f, PrincipalSpectrum(1.f), 1.f, 1.f, ior, distribution);
        isect->bsdf->add(trans);
    }

private:
    float alpha, ior;
};

class SmoothDielectricMaterial : public Material {
public:
    explicit SmoothDielectricMaterial(float ior) : ior(ior) {}
    void compute_scattering_functions(SurfaceInteraction *isect) const override {
        isect->bsdf = std::make_shared<BSDF>(*isect, ior);
        std::unique_ptr<BxDF> lobe =
            std::make_unique<FresnelSpecularBXDF>(PrincipalSpectrum(1.f), PrincipalSpectrum(1.f), 1.f, ior);
        isect->bsdf->add(lobe);
    }

private:
    float ior;
};

int dump_tables(const char *out) {
    InitializeSpectrals();
    FILE *f = fopen(out, "wb");
    if (!f) return 2;
    int32_t counts[2] = {nCIESamples, nRGB2SpectSamples};
    fwrite(counts, sizeof(int32_t), 2, f);
    fwrite(&CIE_Y_Integral, sizeof(float), 1, f);
    fwrite(CIE_Wavelength, sizeof(float), nCIESamples, f);
    fwrite(CIE_X, sizeof(float), nCIESamples, f);
    fwrite(CIE_Y, sizeof(float), nCIESamples, f);
    fwrite(CIE_Z, sizeof(float), nCIESamples, f);
    fwrite(RGB2SpectLambda, sizeof(float), nRGB2SpectSamples, f);
    const float *refl[7] = {RGBRefl2SpectWhite, RGBRefl2SpectCyan, RGBRefl2SpectMagenta, RGBRefl2SpectYellow,
                            RGBRefl2SpectRed, RGBRefl2SpectGreen, RGBRefl2SpectBlue};
    const float *illum[7] = {RGBIllum2SpectWhite, RGBIllum2SpectCyan, RGBIllum2SpectMagenta, RGBIllum2SpectYellow,
                             RGBIllum2SpectRed, RGBIllum2SpectGreen, RGBIllum2SpectBlue};
    for (auto *p : refl) fwrite(p, sizeof(float), nRGB2SpectSamples, f);
    for (auto *p : illum) fwrite(p, sizeof(float), nRGB2SpectSamples, f);
    const PrincipalSpectrum *binned[17] = {&X, &Y, &Z,
                                           &rgbRefl2SpectWhite, &rgbRefl2SpectCyan, &rgbRefl2SpectMagenta,
                                           &rgbRefl2SpectYellow, &rgbRefl2SpectRed, &rgbRefl2SpectGreen,
                                           &rgbRefl2SpectBlue,
                                           &rgbIllum2SpectWhite, &rgbIllum2SpectCyan, &rgbIllum2SpectMagenta,
                                           &rgbIllum2SpectYellow, &rgbIllum2SpectRed, &rgbIllum2SpectGreen,
                                           &rgbIllum2SpectBlue};
    for (auto *s : binned) fwrite(s->c, sizeof(float), nSpectralSamples, f);
    /* from_reflectance_rgb of the Cornell albedos and to_xyz of a constant spectrum */
    const float rgbs[4][3] = {{0.725f, 0.725f, 0.725f}, {0.63f, 0.065f, 0.05f}, {0.14f, 0.45f, 0.091f}, {0.2f, 0.9f, 0.5f}};
    for (auto &c : rgbs) {
        PrincipalSpectrum s = from_reflectance_rgb(Vector3f(c[0], c[1], c[2]));
        fwrite(s.c, sizeof(float), nSpectralSamples, f);
    }
    Vector3f xyz = to_xyz(PrincipalSpectrum(1.f));
    float x3[3] = {xyz.x, xyz.y, xyz.z};
    fwrite(x3, sizeof(float), 3, f);
    fclose(f);
    return 0;
}

// the raw curves in GetMetalCoefficientsFromForge's order, then InitializeForge's 60-bin eta / k
int dump_metals(const char *out) {
    FILE *f = fopen(out, "wb");
    if (!f) return 2;
    const int ns[9] = {Gold_nSamples, Copper_nSamples, Silver_nSamples, Aluminium_nSamples, Beryllium_nSamples,
                       Chromium_nSamples, Mercury_nSamples, Iridium_nSamples, Lithium_nSamples};
    const float *lam[9] = {Gold_Lambda, Copper_Lambda, Silver_Lambda, Aluminium_Lambda, Beryllium_Lambda,
                           Chromium_Lambda, Mercury_Lambda, Iridium_Lambda, Lithium_Lambda};
    const float *eta[9] = {Gold_Eta, Copper_Eta, Silver_Eta, Aluminium_Eta, Beryllium_Eta,
                           Chromium_Eta, Mercury_Eta, Iridium_Eta, Lithium_Eta};
    const float *kk[9] = {Gold_K, Copper_K, Silver_K, Aluminium_K, Beryllium_K,
                          Chromium_K, Mercury_K, Iridium_K, Lithium_K};
    int32_t n9[9];
    for (int m = 0; m < 9; ++m) n9[m] = ns[m];
    fwrite(n9, sizeof(int32_t), 9, f);
    for (int m = 0; m < 9; ++m) {
        fwrite(lam[m], sizeof(float), ns[m], f);
        fwrite(eta[m], sizeof(float), ns[m], f);
        fwrite(kk[m], sizeof(float), ns[m], f);
    }
    InitializeForge();
    for (int m = 0; m < 9; ++m) {
        const std::pair<PrincipalSpectrum, PrincipalSpectrum> p = GetMetalCoefficientsFromForge(m);
        fwrite(p.first.c, sizeof(float), nSpectralSamples, f);
        fwrite(p.second.c, sizeof(float), nSpectralSamples, f);
    }
    fclose(f);
    return 0;
}

int dump_pcg(const char *out) {
    FILE *f = fopen(out, "wb");
    if (!f) return 2;
    const uint64_t seeds[5][2] = {{0, 1}, {1, 1}, {12345, 1}, {42, 54}, {65535, 1}};
    for (auto &s : seeds) {
        pcg32 r(s[0], s[1]);
        uint32_t v[16];
        for (auto &x : v) x = r.nextUInt();
        fwrite(v, sizeof(uint32_t), 16, f);
    }
    const int64_t advs[3] = {1, 1 << 16, 5 << 16};
    for (int64_t a : advs) {
        pcg32 r(7, 1);
        r.advance(a);
        uint32_t v[8];
        for (auto &x : v) x = r.nextUInt();
        fwrite(v, sizeof(uint32_t), 8, f);
    }
    pcg32 r(3, 1);
    float fl[8];
    for (auto &x : fl) x = r.nextFloat();
    fwrite(fl, sizeof(float), 8, f);
    fclose(f);
    return 0;
}

int render(const char *scene_path, const char *out_path, bool forge) {
    FILE *f = fopen(scene_path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", scene_path); return 2; }
    SceneFileHeader h;
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, "FLSCENE2", 8) != 0) {
        fprintf(stderr, "bad scene file\n");
        return 2;
    }
    std::vector<float> verts;
    std::vector<uint32_t> tri_mat, pixels;
    std::vector<fl_material> mats;
    std::vector<fl_light> lights;
    bool ok = read_n(f, verts, (size_t)h.n_tri * 9) && read_n(f, tri_mat, h.n_tri) && read_n(f, mats, h.n_mat) &&
              read_n(f, lights, h.n_light) && read_n(f, pixels, h.n_pixels);
    // optional trailer: the StandardSurfaceMaterial parameters of FL_MAT_STANDARD materials
    std::vector<fl_standard_surface> stds;
    uint32_t n_std = 0;
    if (ok && fread(&n_std, sizeof(n_std), 1, f) == 1) ok = read_n(f, stds, n_std);
    // optional: texture coordinates (6 per triangle) and RGB images, each written out as a
    // binary PPM for the reference's own ImageMapTexture (stbi_load) to read
    uint32_t has_uvs = 0, n_img = 0;
    std::vector<std::string> image_paths;
    std::vector<std::shared_ptr<Texture<float>>> heights;
    if (ok && fread(&has_uvs, sizeof(has_uvs), 1, f) == 1) {
        if (has_uvs) ok = read_n(f, ref_shim::g_uvs, (size_t)h.n_tri * 6);
        if (ok && fread(&n_img, sizeof(n_img), 1, f) == 1) {
            for (uint32_t i = 0; ok && i < n_img; ++i) {
                int32_t wh[2];
                std::vector<uint8_t> px;
                ok = fread(wh, sizeof(int32_t), 2, f) == 2 && wh[0] > 0 && wh[1] > 0 &&
                     read_n(f, px, (size_t)wh[0] * wh[1] * 3);
                if (!ok) break;
                const std::string path = std::string(out_path) + ".tex" + std::to_string(i) + ".ppm";
                FILE *o = fopen(path.c_str(), "wb");
                if (!o) { ok = false; break; }
                fprintf(o, "P6\n%d %d\n255\n", wh[0], wh[1]);
                fwrite(px.data(), 1, px.size(), o);
                fclose(o);
                image_paths.push_back(path);
                heights.push_back(std::make_shared<RedChannelTexture>(wh[0], wh[1], std::move(px)));
            }
        }
    }
    fclose(f);
    if (!ok) { fprintf(stderr, "truncated scene file\n"); return 2; }
    std::vector<std::shared_ptr<Texture<PrincipalSpectrum>>> images;
    for (const std::string &p : image_paths) images.push_back(std::make_shared<ImageMapTexture>(p.c_str()));
    if (h.spectral_mode != FL_SPECTRAL_BINS60) {
        fprintf(stderr, "the reference integrator only has 60-bin spectra\n");
        return 2;
    }

    InitializeSpectrals();
    if (forge) InitializeForge();

    std::vector<std::shared_ptr<Material>> materials;
    for (const auto &m : mats) {
        const float alpha = m.roughness * m.roughness;
        if (m.type == FL_MAT_LAMBERT && m.texture > 0 && (size_t)m.texture <= images.size()) {
            materials.push_back(std::make_shared<LambertMaterial>(images[m.texture - 1]));
        } else if (m.type == FL_MAT_LAMBERT) {
            PrincipalSpectrum r = from_reflectance_rgb(Vector3f(m.rgb[0], m.rgb[1], m.rgb[2]));
            materials.push_back(
                std::make_shared<LambertMaterial>(std::make_shared<ConstantTexture<PrincipalSpectrum>>(r)));
        } else if (m.type == FL_MAT_CONDUCTOR) {
            materials.push_back(std::make_shared<ConductorMaterial>(alpha, m.eta, m.k));
        } else if (m.type == FL_MAT_ROUGH_DIELECTRIC) {
            materials.push_back(std::make_shared<RoughDielectricMaterial>(alpha, m.eta));
        } else if (m.type == FL_MAT_SMOOTH_DIELECTRIC) {
            materials.push_back(std::make_shared<SmoothDielectricMaterial>(m.eta));
        } else if (m.type == FL_MAT_STANDARD && m.standard >= 0 && (uint32_t)m.standard < stds.size()) {
            // the reference's own StandardSurfaceMaterial with constant textures
            const fl_standard_surface &p = stds[m.standard];
            auto spec = [](const float c[3]) {
                return std::make_shared<ConstantTexture<PrincipalSpectrum>>(from_reflectance_rgb(Vector3f(c[0], c[1], c[2])));
            };
            auto flt = [](float v) { return std::make_shared<ConstantTexture<float>>(v); };
            materials.push_back(std::make_shared<StandardSurfaceMaterial>(
                p.kd_weight,
                (p.kd_texture > 0 && (size_t)p.kd_texture <= images.size()) ? images[p.kd_texture - 1] : spec(p.kd),
                flt(p.kd_roughness), p.ks_weight, spec(p.ks), flt(p.ks_roughness),
                flt(p.ks_anisotropic), p.fresnel_type, p.ks_ior, p.metal_type, p.sheen_weight, spec(p.sheen_color),
                flt(p.sheen_roughness), p.kt_weight, spec(p.kt), p.coat_weight, spec(p.coat_color), p.coat_ior,
                p.coat_gloss, p.thin_film_thickness, p.thin_film_ior, p.thin_walled != 0,
                (p.bump_texture > 0 && (size_t)p.bump_texture <= heights.size()) ? heights[p.bump_texture - 1]
                                                                                   : nullptr));
        } else {
            fprintf(stderr, "unknown material type\n");
            return 2;
        }
    }
    std::vector<std::shared_ptr<Shape>> shapes(h.n_tri);
    for (uint32_t i = 0; i < h.n_tri; ++i) {
        const float *v = &verts[9 * (size_t)i];
        shapes[i] = std::make_shared<Triangle>(TriangleEntity(Vector3f(v[0], v[1], v[2])),
                                               TriangleEntity(Vector3f(v[3], v[4], v[5])),
                                               TriangleEntity(Vector3f(v[6], v[7], v[8])), false);
    }
    std::vector<std::shared_ptr<AreaIlluminant>> tri_light(h.n_tri);
    std::vector<std::shared_ptr<Illuminant>> illuminants;
    for (const auto &l : lights) {
        if (l.type == FL_LIGHT_POINT || l.type == FL_LIGHT_SPOT || l.type == FL_LIGHT_DIRECTIONAL) {
            // the reference's delta lights, colour 1 times intensity, quadratic decay
            const Vector3f dir(l.direction[0], l.direction[1], l.direction[2]);
            if (l.type == FL_LIGHT_POINT)
                illuminants.push_back(std::make_shared<PointIlluminant>(
                    translate(l.center[0], l.center[1], l.center[2]), PrincipalSpectrum(1.f), l.radiance, (short)2,
                    PrincipalSpectrum(0.f)));
            else if (l.type == FL_LIGHT_SPOT)
                illuminants.push_back(std::make_shared<SpotIlluminant>(
                    translate(l.center[0], l.center[1], l.center[2]), dir, l.cone_angle, l.penumbra_angle, true, false,
                    PrincipalSpectrum(1.f), l.radiance, (short)2, PrincipalSpectrum(0.f)));
            else
                // an identity transform: a default-constructed Transform is the zero matrix
                illuminants.push_back(std::make_shared<DirectionalIlluminant>(
                    translate(0.f, 0.f, 0.f), dir, PrincipalSpectrum(1.f), l.radiance, PrincipalSpectrum(0.f)));
            continue;
        }
        if (l.type != FL_LIGHT_TRIANGLE || l.tri >= h.n_tri) {
            fprintf(stderr, "harness supports triangle area lights and the delta lights only\n");
            return 2;
        }
        auto al = std::make_shared<DiffuseAreaIlluminant>(Transform(), PrincipalSpectrum(1.f), l.radiance, (short)2,
                                                          PrincipalSpectrum(0.f), shapes[l.tri]);
        tri_light[l.tri] = al;
        illuminants.push_back(al);
    }
    std::vector<std::shared_ptr<GeometricPrimitive>> prims(h.n_tri);
    SceneGeometry geom;
    auto mesh = std::make_shared<TriangleMesh>();
    ref_shim::g_primitives.assign(h.n_tri, nullptr);
    for (uint32_t i = 0; i < h.n_tri; ++i) {
        prims[i] = std::make_shared<GeometricPrimitive>(shapes[i], materials[tri_mat[i]], tri_light[i]);
        ref_shim::g_primitives[i] = prims[i].get();
        auto bt = std::make_shared<BasicTriangle>();
        const float *v = &verts[9 * (size_t)i];
        bt->v1 = Vector3f(v[0], v[1], v[2]);
        bt->v2 = Vector3f(v[3], v[4], v[5]);
        bt->v3 = Vector3f(v[6], v[7], v[8]);
        mesh->triangles.push_back(bt);
    }
    geom.triangleMeshes.push_back(mesh);
    Scene scene(geom, illuminants);

    const fl_camera &c = h.cam;
    if (c.aperture != 0.f) {
        // random_point_on_lens (cameras/physical.cpp:4-10) never returns for lens samples
        // outside the unit disk: the reference can only render a pinhole here
        fprintf(stderr, "the reference's lens sampler does not terminate: aperture must be 0\n");
        return 2;
    }
    PhysicalCamera camera(Vector3f(c.position[0], c.position[1], c.position[2]),
                          Vector3f(c.look_at[0], c.look_at[1], c.look_at[2]), c.width, c.height, c.vfov_deg, 0.f, 0.f,
                          0.f, Vector3f(c.up[0], c.up[1], c.up[2]), true);
    RenderParams rp{(int)h.spp, (int)h.diffuse_depth, (int)h.reflection_depth, (int)h.transmission_depth};
    PathIntegrator integrator(rp, h.rr_threshold);

    const uint32_t W = (uint32_t)c.width, H = (uint32_t)c.height;
    const uint32_t total = h.n_pixels ? h.n_pixels : W * H;
    std::vector<double> film((size_t)W * H * 3, 0.0);
    std::atomic<uint32_t> next{0};
    unsigned nth = h.nthreads ? h.nthreads : std::thread::hardware_concurrency();
    if (nth == 0) nth = 1;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> threads;
    for (unsigned k = 0; k < nth; ++k) {
        threads.emplace_back([&]() {
            PCG32Sampler sampler;
            for (;;) {
                uint32_t start = next.fetch_add(64);
                if (start >= total) break;
                uint32_t end = std::min(total, start + 64);
                for (uint32_t q = start; q < end; ++q) {
                    uint32_t pixel = h.n_pixels ? pixels[q] : q;
                    uint32_t px = pixel % W, py = pixel / W;
                    double acc[3] = {0, 0, 0};
                    for (uint32_t s = 0; s < h.spp; ++s) {
                        sampler.reset(pixel, (uint64_t)h.sample_offset + s);
                        float ux = sampler.get_1d();
                        float uy = sampler.get_1d();
                        (void)sampler.get_1d(); /* hero-wavelength draw, unused by 60 bins */
                        float sx = ((float)px + ux) / (float)W;
                        float sy = ((float)(H - 1u - py) + uy) / (float)H;
                        Ray ray = camera.awaken_ray(Vector2f(sx, sy), Vector2f(0.5f, 0.5f));
                        PrincipalSpectrum L = integrator.Li(ray, scene, sampler, 0);
                        Vector3f xyz = to_xyz(L);
                        acc[0] += xyz.x;
                        acc[1] += xyz.y;
                        acc[2] += xyz.z;
                    }
                    film[3 * (size_t)pixel + 0] = acc[0];
                    film[3 * (size_t)pixel + 1] = acc[1];
                    film[3 * (size_t)pixel + 2] = acc[2];
                }
            }
        });
    }
    for (auto &t : threads) t.join();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    FILE *o = fopen(out_path, "wb");
    if (!o) return 2;
    fwrite(film.data(), sizeof(double), film.size(), o);
    fclose(o);
    printf("{\"pixels\": %u, \"spp\": %u, \"threads\": %u, \"seconds\": %.6f}\n", total, h.spp, nth, secs);
    return 0;
}

} // namespace

int main(int argc, char **argv) {
    if (argc == 3 && strcmp(argv[1], "--tables") == 0) return dump_tables(argv[2]);
    if (argc == 3 && strcmp(argv[1], "--pcg") == 0) return dump_pcg(argv[2]);
    if (argc == 3 && strcmp(argv[1], "--metals") == 0) return dump_metals(argv[2]);
    if (argc == 3) return render(argv[1], argv[2], false);
    if (argc == 4 && strcmp(argv[3], "--forge") == 0) return render(argv[1], argv[2], true);
    fprintf(stderr, "usage: ref_render SCENE.bin OUT.bin [--forge] | --tables OUT.bin | --metals OUT.bin | --pcg OUT.bin\n");
    return 1;
}
