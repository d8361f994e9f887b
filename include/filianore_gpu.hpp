// filianore_gpu.hpp: C++ host adapter over the C ABI of filianore_gpu.h.
//
// It mirrors the reference's classes on this path, so that code written against
// filianore-core reads the same against the GPU backend:
//   SceneGeometry / TriangleMesh / BasicTriangle   src/filianore/bvh/bvh.h:11-21
//   BVH (initialize, initialize_scene_geometry,     src/filianore/bvh/bvh.h:23-45,
//        add_triangle_mesh, finalise, intersect,    src/filianore/bvh/bvh.cpp:7-88
//        intersect_p, clean_up)
//   Scene (geometry + illuminants, owns its BVH)   src/filianore/core/scene.h:12-27
//   RenderParams                                    src/filianore/core/renderparams.h:5-10
//   PathIntegrator(RenderParams, rrThreshold)       src/filianore/integrators/pathintegrator.h:9-22
//     with Li(ray, scene, sampler, depth)           src/filianore/integrators/integrator.h:17-18
//   PhysicalCamera (position, look-at, up, fov)     src/filianore/cameras/physical.h:11-43
//     with awaken_ray                               src/filianore/cameras/physical.cpp:12-22
//   PCG32Sampler (a Sampler over pcg32)             src/filianore/sampling/sampler.h:10-19, src/ext/pcg32.h
// The types are this library's own (plain structs), not the reference's: a maintainer
// converts at the boundary, as shown in the integration notes.
//
// Conventions kept from the reference: intersect / intersect_p return bool (hit or not)
// and shrink ray.tMax on a hit; nothing throws. A failure of the library (no device, out of
// memory) makes the call report a miss or false and leaves the message in last_error().
// The GPU's granularity: PathIntegrator renders whole images (render), the replacement of
// the application's loop over Integrator::Li; Li itself is there for single rays and batches
// (one device launch sequence per call, so slow per ray).
#ifndef FILIANORE_GPU_HPP
#define FILIANORE_GPU_HPP

#include <cmath>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "filianore_gpu.h"

namespace filianore_gpu {

struct Vector3f {
    float x = 0.f, y = 0.f, z = 0.f;
};

struct Vector2f {
    float x = 0.f, y = 0.f;
};

// A triangle of the soup, with the texture coordinates of its vertices (TriangleEntity::uv).
struct BasicTriangle {
    Vector3f v1, v2, v3;
    Vector2f uv1, uv2, uv3;
};

// One mesh of the soup. `material` indexes Scene's materials (the reference attaches a
// Material per GeometricPrimitive instead).
struct TriangleMesh {
    std::vector<std::shared_ptr<BasicTriangle>> triangles;
    uint32_t material = 0;
};

struct SceneGeometry {
    std::vector<std::shared_ptr<TriangleMesh>> triangleMeshes;
};

struct Ray {
    Vector3f origin, dir;
    float tMin = 0.f;
    mutable float tMax = std::numeric_limits<float>::infinity();  // shrunk by intersect, as in the reference
};

// The part of the reference's SurfaceInteraction the hit provides: distance, point, the
// geometric normal normalize(cross(v2 - v1, v3 - v1)), the primitive (soup index) and
// embree's barycentrics.
struct SurfaceInteraction {
    float t = 0.f;
    Vector3f p, n;
    int primitive = -1;
    float u = 0.f, v = 0.f;
};

struct RenderParams {
    int samples = 1;
    int diffuseRayDepth = 8;
    int reflectionRayDepth = 8;
    int transmissionRayDepth = 8;
};

// The reference's 60-bin spectrum (color/principalspectrum.h:7-21), as Li returns it.
struct PrincipalSpectrum {
    float c[60] = {};
};

// A Sampler over O'Neill's PCG32 (the generator of src/ext/pcg32.h), the sampler the GPU
// renders with: seed(pixel, 1) per pixel, get_1d = nextFloat, get_2d = (get_1d, get_1d).
// Li continues the sampler's stream on the device, which supports the default stream
// (initseq 1) only.
class PCG32Sampler {
public:
    uint64_t state = 0x853c49e6748fea9bULL, inc = 0xda3e39cb94b95bdbULL;
    void seed(uint64_t initstate, uint64_t initseq = 1u) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        next_uint();
        state += initstate;
        next_uint();
    }
    uint32_t next_uint() {
        const uint64_t old = state;
        state = old * 0x5851f42d4c957f2dULL + inc;
        const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
    }
    float get_1d() {
        union {
            uint32_t u;
            float f;
        } x;
        x.u = (next_uint() >> 9) | 0x3f800000u;
        return x.f - 1.0f;
    }
    Vector2f get_2d() {
        const float a = get_1d();
        const float b = get_1d();
        return Vector2f{a, b};
    }
    // jump ahead by delta draws (Brown's method, as pcg32::advance)
    void advance(uint64_t delta) {
        uint64_t cur_mult = 0x5851f42d4c957f2dULL, cur_plus = inc, acc_mult = 1u, acc_plus = 0u;
        while (delta > 0) {
            if (delta & 1) {
                acc_mult *= cur_mult;
                acc_plus = acc_plus * cur_mult + cur_plus;
            }
            cur_plus = (cur_mult + 1) * cur_plus;
            cur_mult *= cur_mult;
            delta /= 2;
        }
        state = acc_mult * state + acc_plus;
    }
};

struct PhysicalCamera {
    Vector3f position, lookAt, up{0.f, 1.f, 0.f};
    float fov = 40.f;  // vertical, degrees
    int xRes = 256, yRes = 256;
    float aperture = 0.f;  // lens diameter, focused at lookAt (0: pinhole)

    // PhysicalCamera::awaken_ray (cameras/physical.cpp:12-22) for a pinhole, with the
    // constructor's basis (physical.h:11-43, flipCameraDirection = true) in the reference's
    // operation order: the ray the device renders for camera sample s (x, y in [0, 1]).
    Ray awaken_ray(const Vector2f &s) const {
        const Vector3f pos = position;
        const float focusDistance = length(sub(pos, lookAt));
        const float theta = fov * 3.14159265358979323846f / 180.f;
        const float halfHeight = std::tan(theta / 2.f);
        const float aspect = (float)xRes / (float)yRes;
        const float halfWidth = aspect * halfHeight;
        Vector3f w = normalize(sub(pos, lookAt));
        w = mul(w, -1.f);
        const Vector3f u = normalize(cross(up, w));
        const Vector3f v = cross(w, u);
        w = mul(w, -1.f);
        const Vector3f lowerLeft =
            sub(sub(sub(pos, mul(mul(u, halfWidth), focusDistance)), mul(mul(v, focusDistance), halfHeight)),
                mul(w, focusDistance));
        const Vector3f horizontal = mul(mul(mul(u, 2.f), halfWidth), focusDistance);
        const Vector3f vertical = mul(mul(mul(v, 2.f), halfHeight), focusDistance);
        // random_point_on_lens((0.5, 0.5)) * lensRadius with lensRadius 0 for a pinhole
        const Vector3f rd = mul(sub(mul(Vector3f{0.5f, 0.5f, 0.f}, 2.f), Vector3f{1.f, 1.f, 0.f}), 0.f);
        const Vector3f offset = add(mul(u, rd.x), mul(v, rd.y));
        Ray r;
        r.origin = add(pos, offset);
        r.dir = normalize(sub(sub(add(add(lowerLeft, mul(horizontal, s.x)), mul(vertical, s.y)), pos), offset));
        r.tMin = 0.f;  // time0 + s.x (time1 - time0) with no shutter interval
        return r;
    }
    // The render loop's camera ray of pixel (px, py), row 0 at the top: the sampler draws
    // (ux, uy) and then the hero wavelength's number, as the device does.
    Ray pixel_ray(int px, int py, PCG32Sampler &sampler, float *u_lambda = nullptr) const {
        const float ux = sampler.get_1d(), uy = sampler.get_1d();
        const float ul = sampler.get_1d();
        if (u_lambda) *u_lambda = ul;
        const float sx = ((float)px + ux) / (float)xRes;
        const float sy = ((float)(yRes - 1 - py) + uy) / (float)yRes;
        return awaken_ray(Vector2f{sx, sy});
    }

private:
    // maths/geometry.h's operations: products as s * x, cross in double, normalize by the
    // reciprocal of the length
    static Vector3f add(Vector3f a, Vector3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
    static Vector3f sub(Vector3f a, Vector3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    static Vector3f mul(Vector3f a, float s) { return {s * a.x, s * a.y, s * a.z}; }
    static float length(Vector3f a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
    static Vector3f normalize(Vector3f a) {
        const float inv = 1.f / length(a);
        return {a.x * inv, a.y * inv, a.z * inv};
    }
    static Vector3f cross(Vector3f a, Vector3f b) {
        const double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
        return {(float)((ay * bz) - (az * by)), (float)((az * bx) - (ax * bz)), (float)((ax * by) - (ay * bx))};
    }
};

// An illuminant: a triangle of the soup (DiffuseAreaIlluminant), a point, spot or
// directional light (PointIlluminant, SpotIlluminant, DirectionalIlluminant), an analytic
// sphere or a constant environment (the last two new in this backend).
struct Illuminant {
    int type = FL_LIGHT_TRIANGLE;
    uint32_t triangle = 0;
    float radiance = 0.f;  // color * intensity
    Vector3f center;       // sphere centre, point / spot position
    float radius = 0.f;
    Vector3f direction{0.f, -1.f, 0.f};  // spot axis, or the direction a directional light travels
    float cone_angle = 0.f, penumbra_angle = 0.f;  // spot, radians from the axis
};

// StandardSurfaceMaterial: its parameters are standard_surfaces[index] of the Scene
inline fl_material StandardSurfaceMaterial(int32_t index) {
    fl_material m{};
    m.type = FL_MAT_STANDARD;
    m.standard = index;
    return m;
}

inline fl_material LambertMaterial(float r, float g, float b) {
    fl_material m{};
    m.type = FL_MAT_LAMBERT;
    m.rgb[0] = r;
    m.rgb[1] = g;
    m.rgb[2] = b;
    return m;
}

inline std::string status_text(const fl_context *ctx, fl_status st) {
    char buf[512] = {0};
    fl_last_error(ctx, buf, sizeof(buf));
    return std::string(fl_status_string(st)) + (buf[0] ? std::string(": ") + buf : std::string());
}

// The device and the spectral tables (the reference's InitializeSpectrals()).
class Context {
public:
    Context(int device, const fl_spectral_tables &tables) {
        st_ = fl_context_create(device, &tables, &ctx_);
        if (st_ != FL_OK) error_ = status_text(nullptr, st_);
    }
    ~Context() {
        if (ctx_) fl_context_destroy(ctx_);
    }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    bool ok() const { return ctx_ != nullptr; }
    fl_context *get() const { return ctx_; }
    const std::string &last_error() const { return error_; }

private:
    fl_context *ctx_ = nullptr;
    fl_status st_ = FL_OK;
    std::string error_;
};

// The acceleration structure (the reference's BVH over embree).
class BVH {
public:
    BVH() = default;
    ~BVH() { clean_up(); }
    BVH(const BVH &) = delete;
    BVH &operator=(const BVH &) = delete;

    void initialize(Context &ctx) { ctx_ = &ctx; }
    void clean_up() {
        if (scene_) fl_scene_destroy(scene_);
        scene_ = nullptr;
    }

    // Triangle ids are insertion order across meshes, as embree's geomIDs.
    void initialize_scene_geometry(const SceneGeometry &geometry) {
        for (const auto &mesh : geometry.triangleMeshes)
            for (const auto &tri : mesh->triangles) add_triangle_mesh(tri, mesh->material);
    }
    void add_triangle_mesh(const std::shared_ptr<BasicTriangle> &tri, uint32_t material = 0) {
        const BasicTriangle &t = *tri;
        const float v[9] = {t.v1.x, t.v1.y, t.v1.z, t.v2.x, t.v2.y, t.v2.z, t.v3.x, t.v3.y, t.v3.z};
        soup_.insert(soup_.end(), v, v + 9);
        tri_material_.push_back(material);
        const float uv[6] = {t.uv1.x, t.uv1.y, t.uv2.x, t.uv2.y, t.uv3.x, t.uv3.y};
        uvs_.insert(uvs_.end(), uv, uv + 6);
        for (float c : uv) has_uvs_ = has_uvs_ || c != 0.f;
    }
    // Builds the device BVH (embree's rtcCommitScene). Returns false on failure. `images`
    // are the ImageMapTextures the materials name (their pixels are copied during the call).
    bool finalise(const std::vector<fl_material> &materials, const std::vector<fl_light> &lights,
                  const std::vector<fl_standard_surface> &standard_surfaces = {},
                  const std::vector<fl_image> &images = {}) {
        clean_up();
        if (!ctx_ || !ctx_->ok()) {
            error_ = "BVH::finalise without a valid context";
            return false;
        }
        fl_scene_desc d{};
        d.verts = soup_.data();
        d.n_tri = (uint32_t)(soup_.size() / 9);
        d.tri_material = tri_material_.data();
        d.materials = materials.data();
        d.n_materials = (uint32_t)materials.size();
        d.lights = lights.data();
        d.n_lights = (uint32_t)lights.size();
        d.standard_surfaces = standard_surfaces.empty() ? nullptr : standard_surfaces.data();
        d.n_standard_surfaces = (uint32_t)standard_surfaces.size();
        d.uvs = has_uvs_ ? uvs_.data() : nullptr;  // all zero: every hit at uv (0, 0) either way
        d.images = images.empty() ? nullptr : images.data();
        d.n_images = (uint32_t)images.size();
        const fl_status st = fl_scene_create(ctx_->get(), &d, &scene_);
        if (st != FL_OK) {
            error_ = status_text(ctx_->get(), st);
            scene_ = nullptr;
            return false;
        }
        return true;
    }

    // One ray (the reference's per-ray call); renderers that batch use trace().
    bool intersect(const Ray &ray, SurfaceInteraction *isect) const {
        SurfaceInteraction h;
        if (!trace(&ray, 1, &h) || h.primitive < 0) return false;
        if (isect) *isect = h;
        ray.tMax = h.t;
        return true;
    }
    bool intersect_p(const Ray &ray) const {
        if (!scene_) return false;
        const float o[4] = {ray.origin.x, ray.origin.y, ray.origin.z, ray.tMin};
        const float d[4] = {ray.dir.x, ray.dir.y, ray.dir.z, ray.tMax};
        uint8_t occ = 0;
        if (fl_trace_occluded(scene_, o, d, 1, &occ, FL_MEM_HOST, nullptr) != FL_OK) return false;
        return occ != 0;
    }
    // Closest hits of n rays in one call; returns false when the library fails.
    bool trace(const Ray *rays, uint32_t n, SurfaceInteraction *out) const {
        if (!scene_) return false;
        std::vector<float> o(4 * (size_t)n), d(4 * (size_t)n);
        for (uint32_t i = 0; i < n; ++i) {
            const Ray &r = rays[i];
            o[4 * i] = r.origin.x, o[4 * i + 1] = r.origin.y, o[4 * i + 2] = r.origin.z, o[4 * i + 3] = r.tMin;
            d[4 * i] = r.dir.x, d[4 * i + 1] = r.dir.y, d[4 * i + 2] = r.dir.z, d[4 * i + 3] = r.tMax;
        }
        std::vector<fl_hit> hits(n);
        if (fl_trace_closest(scene_, o.data(), d.data(), n, hits.data(), FL_MEM_HOST, nullptr) != FL_OK) return false;
        for (uint32_t i = 0; i < n; ++i) {
            SurfaceInteraction &s = out[i];
            s = SurfaceInteraction{};
            s.primitive = hits[i].id;
            if (hits[i].id < 0) continue;
            const Ray &r = rays[i];
            s.t = hits[i].t;
            s.u = hits[i].u;
            s.v = hits[i].v;
            s.p = Vector3f{r.origin.x + r.dir.x * s.t, r.origin.y + r.dir.y * s.t, r.origin.z + r.dir.z * s.t};
            const float *v = &soup_[9 * (size_t)hits[i].id];
            const float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
            const float e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
            Vector3f n{e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            const float len = std::sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
            if (len > 0.f) n = Vector3f{n.x / len, n.y / len, n.z / len};
            s.n = n;
        }
        return true;
    }

    fl_scene *get() const { return scene_; }
    size_t triangle_count() const { return soup_.size() / 9; }
    const std::string &last_error() const { return error_; }

private:
    Context *ctx_ = nullptr;
    fl_scene *scene_ = nullptr;
    std::vector<float> soup_;
    std::vector<uint32_t> tri_material_;
    std::vector<float> uvs_;  // 6 per triangle
    bool has_uvs_ = false;
    std::string error_;
};

// Geometry plus illuminants, owning its BVH (the reference's Scene).
class Scene {
public:
    Scene(Context &ctx, const SceneGeometry &geometry, const std::vector<fl_material> &materials,
          const std::vector<Illuminant> &illuminants, const std::vector<fl_standard_surface> &standard_surfaces = {},
          const std::vector<fl_image> &images = {})
        : illuminants(illuminants) {
        bvh.initialize(ctx);
        bvh.initialize_scene_geometry(geometry);
        std::vector<fl_light> lights;
        for (const Illuminant &il : illuminants) {
            fl_light l{};
            l.type = il.type;
            l.tri = il.triangle;
            l.radiance = il.radiance;
            l.radius = il.radius;
            l.center[0] = il.center.x;
            l.center[1] = il.center.y;
            l.center[2] = il.center.z;
            l.direction[0] = il.direction.x;
            l.direction[1] = il.direction.y;
            l.direction[2] = il.direction.z;
            l.cone_angle = il.cone_angle;
            l.penumbra_angle = il.penumbra_angle;
            lights.push_back(l);
        }
        ok_ = bvh.finalise(materials, lights, standard_surfaces, images);
    }
    ~Scene() { bvh.clean_up(); }
    bool ok() const { return ok_; }
    bool intersect(const Ray &ray, SurfaceInteraction *isect) const { return bvh.intersect(ray, isect); }
    bool intersect_p(const Ray &ray) const { return bvh.intersect_p(ray); }

    BVH bvh;
    std::vector<Illuminant> illuminants;

private:
    bool ok_ = false;
};

// The path tracer, with RenderParams' three depths: a path ends at bounce b when the lobe
// it samples there is diffuse and b == diffuseRayDepth, specular or glossy and
// b == reflectionRayDepth, or a transmission and b == transmissionRayDepth
// (pathintegrator.cpp:55-65).
class PathIntegrator {
public:
    explicit PathIntegrator(const RenderParams &renderParams, float rrThreshold = 1.f)
        : renderParams(renderParams), rrThreshold(rrThreshold) {}

    // Renders the camera's image: linear RGB, xRes * yRes * 3 floats, row 0 at the top.
    // spectral_mode: FL_SPECTRAL_BINS60 (the reference's 60 bins) or FL_SPECTRAL_HERO4.
    // Returns false (message in last_error()) when the library fails.
    bool render(const Scene &scene, const PhysicalCamera &camera, std::vector<float> &rgb,
                int spectral_mode = FL_SPECTRAL_BINS60, fl_render_stats *stats = nullptr) const {
        fl_camera cam{};
        cam.position[0] = camera.position.x, cam.position[1] = camera.position.y, cam.position[2] = camera.position.z;
        cam.look_at[0] = camera.lookAt.x, cam.look_at[1] = camera.lookAt.y, cam.look_at[2] = camera.lookAt.z;
        cam.up[0] = camera.up.x, cam.up[1] = camera.up.y, cam.up[2] = camera.up.z;
        cam.vfov_deg = camera.fov;
        cam.aperture = camera.aperture;
        cam.width = camera.xRes;
        cam.height = camera.yRes;
        fl_render_params p = params(spectral_mode);
        p.spp = renderParams.samples;
        rgb.assign((size_t)camera.xRes * camera.yRes * 3, 0.f);
        const fl_status st = fl_render(scene.bvh.get(), &cam, &p, rgb.data(), nullptr, FL_MEM_HOST, stats);
        if (st != FL_OK) {
            error_ = std::string(fl_status_string(st));
            return false;
        }
        return true;
    }

    // Integrator::Li (integrators/integrator.h:18): the radiance along `ray`, the path drawing
    // its numbers from `sampler`, which is left where the path stopped drawing. `depth` is
    // unused, as in the reference. 60 bins; xyz (nullable) receives to_xyz of the result.
    // A miss (no scene, a library failure) returns black and sets last_error().
    PrincipalSpectrum Li(const Ray &ray, const Scene &scene, PCG32Sampler &sampler, int depth = 0,
                         double xyz[3] = nullptr) const {
        PrincipalSpectrum L;
        Li(&ray, 1, scene, &sampler, &L, depth, xyz);
        return L;
    }
    // Li for n rays in one device call: rays[i] with samplers[i] into out[i] (xyz: 3 per ray).
    bool Li(const Ray *rays, uint32_t n, const Scene &scene, PCG32Sampler *samplers, PrincipalSpectrum *out,
            int depth = 0, double *xyz = nullptr) const {
        (void)depth;
        if (!scene.bvh.get()) {
            error_ = "Li without a scene";
            return false;
        }
        std::vector<float> o(4 * (size_t)n), d(4 * (size_t)n);
        std::vector<uint64_t> rng(n), rng_out(n);
        for (uint32_t i = 0; i < n; ++i) {
            if (samplers[i].inc != 3u) {
                error_ = "the device continues the default PCG32 stream (initseq 1) only";
                return false;
            }
            const Ray &r = rays[i];
            o[4 * i] = r.origin.x, o[4 * i + 1] = r.origin.y, o[4 * i + 2] = r.origin.z, o[4 * i + 3] = r.tMin;
            d[4 * i] = r.dir.x, d[4 * i + 1] = r.dir.y, d[4 * i + 2] = r.dir.z, d[4 * i + 3] = r.tMax;
            rng[i] = samplers[i].state;
        }
        const fl_render_params p = params(FL_SPECTRAL_BINS60);
        const fl_status st = fl_li(scene.bvh.get(), &p, o.data(), d.data(), rng.data(), nullptr, n,
                                   reinterpret_cast<float *>(out), rng_out.data(), xyz, FL_MEM_HOST);
        static_assert(sizeof(PrincipalSpectrum) == 60 * sizeof(float), "60 packed floats");
        if (st != FL_OK) {
            error_ = std::string(fl_status_string(st));
            for (uint32_t i = 0; i < n; ++i) out[i] = PrincipalSpectrum{};
            return false;
        }
        for (uint32_t i = 0; i < n; ++i) samplers[i].state = rng_out[i];
        return true;
    }
    const std::string &last_error() const { return error_; }

    const RenderParams renderParams;
    const float rrThreshold;

private:
    fl_render_params params(int spectral_mode) const {
        fl_render_params p{};
        p.spp = 1;
        p.max_depth = renderParams.diffuseRayDepth;
        p.rr_threshold = rrThreshold;
        p.spectral_mode = spectral_mode;
        p.flags = FL_RENDER_LOBE_DEPTHS;
        p.diffuse_depth = renderParams.diffuseRayDepth;
        p.reflection_depth = renderParams.reflectionRayDepth;
        p.transmission_depth = renderParams.transmissionRayDepth;
        return p;
    }
    mutable std::string error_;
};

}  // namespace filianore_gpu

#endif  // FILIANORE_GPU_HPP
