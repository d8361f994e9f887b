// Drives the C++ adapter (include/filianore_gpu.hpp) the way code written against the
// reference's classes would: SceneGeometry of BasicTriangles -> Scene (owning its BVH) ->
// BVH::intersect per ray and BVH::trace in a batch -> PathIntegrator::render, and
// PathIntegrator::Li on the camera rays of PhysicalCamera::awaken_ray with a PCG32Sampler
// per pixel. Inputs and outputs are raw little-endian files written and read by
// tests/test_cpp_adapter.py:
//   adapter_cornell <input> <output>
// input:  spectral tables (n_cie, y integral, lambda/x/y/z, n_rgb, lambda, refl[7], illum[7]),
//         soup (n_tri, 9 floats per triangle, material per triangle), materials, lights,
//         camera, samples, the diffuse / reflection / transmission depths, spectral mode,
//         rays (n, origin/tmin and direction/tmax)
// output: the image (width * height * 3 floats), then per ray: intersect's (hit, id, t,
//         tMax after the call) and trace's (id, t); then for every pixel, sample 0 (the
//         sampler seeded with the pixel index): Li's XYZ (3 doubles) from one batch call, and
//         for the first 16 pixels the XYZ of single-ray Li calls and the sampler state after.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/filianore_gpu.hpp"

using namespace filianore_gpu;

struct Reader {
    FILE *f;
    template <class T> T get() {
        T v{};
        if (fread(&v, sizeof(T), 1, f) != 1) throw 1;
        return v;
    }
    template <class T> std::vector<T> arr(size_t n) {
        std::vector<T> v(n);
        if (n && fread(v.data(), sizeof(T), n, f) != n) throw 1;
        return v;
    }
};

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE *in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    Reader r{in};
    std::vector<float> lam, x, y, z, rl;
    std::vector<float> refl[7], illum[7];
    fl_spectral_tables t{};
    std::vector<fl_material> mats;
    std::vector<fl_light> lights_raw;
    std::vector<fl_standard_surface> standard;
    std::vector<std::vector<uint8_t>> pixels;
    std::vector<fl_image> images;
    fl_camera cam{};
    SceneGeometry geometry;
    int spp = 0, depth_d = 0, depth_r = 0, depth_t = 0, mode = 0;
    std::vector<Ray> rays;
    try {
        const int n_cie = r.get<int32_t>();
        t.cie_y_integral = r.get<float>();
        lam = r.arr<float>(n_cie), x = r.arr<float>(n_cie), y = r.arr<float>(n_cie), z = r.arr<float>(n_cie);
        const int n_rgb = r.get<int32_t>();
        rl = r.arr<float>(n_rgb);
        for (int b = 0; b < 7; ++b) refl[b] = r.arr<float>(n_rgb);
        for (int b = 0; b < 7; ++b) illum[b] = r.arr<float>(n_rgb);
        t.cie_lambda = lam.data(), t.cie_x = x.data(), t.cie_y = y.data(), t.cie_z = z.data(), t.n_cie = n_cie;
        t.rgb2spec_lambda = rl.data(), t.n_rgb2spec = n_rgb;
        for (int b = 0; b < 7; ++b) t.refl[b] = refl[b].data(), t.illum[b] = illum[b].data();
        const uint32_t n_tri = r.get<uint32_t>();
        const std::vector<float> soup = r.arr<float>(9 * (size_t)n_tri);
        const std::vector<uint32_t> tri_mat = r.arr<uint32_t>(n_tri);
        mats = r.arr<fl_material>(r.get<uint32_t>());
        lights_raw = r.arr<fl_light>(r.get<uint32_t>());
        cam = r.get<fl_camera>();
        spp = r.get<int32_t>(), depth_d = r.get<int32_t>(), depth_r = r.get<int32_t>(), depth_t = r.get<int32_t>();
        mode = r.get<int32_t>();
        const uint32_t n_rays = r.get<uint32_t>();
        const std::vector<float> org = r.arr<float>(4 * (size_t)n_rays), dir = r.arr<float>(4 * (size_t)n_rays);
        standard = r.arr<fl_standard_surface>(r.get<uint32_t>());
        // texture coordinates (6 per triangle, all zero when the scene has none) and images
        const std::vector<float> uvs = r.arr<float>(6 * (size_t)n_tri);
        const uint32_t n_img = r.get<uint32_t>();
        for (uint32_t i = 0; i < n_img; ++i) {
            const int32_t w = r.get<int32_t>(), h = r.get<int32_t>();
            pixels.push_back(r.arr<uint8_t>(3 * (size_t)w * (size_t)h));
            images.push_back(fl_image{w, h, nullptr});
        }
        for (size_t i = 0; i < images.size(); ++i) images[i].rgb = pixels[i].data();
        // one mesh per triangle keeps the per-triangle materials and the soup order
        for (uint32_t i = 0; i < n_tri; ++i) {
            auto mesh = std::make_shared<TriangleMesh>();
            auto tri = std::make_shared<BasicTriangle>();
            const float *v = &soup[9 * (size_t)i];
            tri->v1 = {v[0], v[1], v[2]}, tri->v2 = {v[3], v[4], v[5]}, tri->v3 = {v[6], v[7], v[8]};
            const float *q = &uvs[6 * (size_t)i];
            tri->uv1 = {q[0], q[1]}, tri->uv2 = {q[2], q[3]}, tri->uv3 = {q[4], q[5]};
            mesh->triangles.push_back(tri);
            mesh->material = tri_mat[i];
            geometry.triangleMeshes.push_back(mesh);
        }
        for (uint32_t i = 0; i < n_rays; ++i) {
            Ray ray;
            ray.origin = {org[4 * i], org[4 * i + 1], org[4 * i + 2]};
            ray.tMin = org[4 * i + 3];
            ray.dir = {dir[4 * i], dir[4 * i + 1], dir[4 * i + 2]};
            ray.tMax = dir[4 * i + 3];
            rays.push_back(ray);
        }
    } catch (int) {
        std::fprintf(stderr, "short input\n");
        return 2;
    }
    std::fclose(in);

    Context ctx(0, t);
    if (!ctx.ok()) {
        std::fprintf(stderr, "context: %s\n", ctx.last_error().c_str());
        return 1;
    }
    std::vector<Illuminant> illuminants;
    for (const fl_light &l : lights_raw) {
        Illuminant il;
        il.type = l.type, il.triangle = l.tri, il.radiance = l.radiance, il.radius = l.radius;
        il.center = {l.center[0], l.center[1], l.center[2]};
        il.direction = {l.direction[0], l.direction[1], l.direction[2]};
        il.cone_angle = l.cone_angle, il.penumbra_angle = l.penumbra_angle;
        illuminants.push_back(il);
    }
    int rc = 0;
    {
        Scene scene(ctx, geometry, mats, illuminants, standard, images);
        if (!scene.ok()) {
            std::fprintf(stderr, "scene: %s\n", scene.bvh.last_error().c_str());
            return 1;
        }
        RenderParams params;
        params.samples = spp;
        params.diffuseRayDepth = depth_d;
        params.reflectionRayDepth = depth_r;
        params.transmissionRayDepth = depth_t;
        PathIntegrator integrator(params);
        PhysicalCamera camera;
        camera.position = {cam.position[0], cam.position[1], cam.position[2]};
        camera.lookAt = {cam.look_at[0], cam.look_at[1], cam.look_at[2]};
        camera.up = {cam.up[0], cam.up[1], cam.up[2]};
        camera.fov = cam.vfov_deg, camera.xRes = cam.width, camera.yRes = cam.height;
        std::vector<float> rgb;
        if (!integrator.render(scene, camera, rgb, mode)) {
            std::fprintf(stderr, "render: %s\n", integrator.last_error().c_str());
            return 1;
        }
        std::vector<SurfaceInteraction> batch(rays.size());
        if (!rays.empty() && !scene.bvh.trace(rays.data(), (uint32_t)rays.size(), batch.data())) rc = 1;
        FILE *out = std::fopen(argv[2], "wb");
        if (!out) return 2;
        std::fwrite(rgb.data(), sizeof(float), rgb.size(), out);
        for (size_t i = 0; i < rays.size(); ++i) {
            SurfaceInteraction si;
            const int32_t hit = scene.intersect(rays[i], &si) ? 1 : 0;  // shrinks rays[i].tMax on a hit
            const int32_t id = hit ? si.primitive : -1;
            const float rec[4] = {(float)hit, (float)id, hit ? si.t : 0.f, rays[i].tMax};
            std::fwrite(rec, sizeof(float), 4, out);
            const float b[2] = {(float)batch[i].primitive, batch[i].t};
            std::fwrite(b, sizeof(float), 2, out);
        }
        // Integrator::Li on every pixel's camera ray (sample 0), in one batch ...
        const int W = camera.xRes, H = camera.yRes;
        std::vector<Ray> cam_rays;
        std::vector<PCG32Sampler> samplers;
        for (int p = 0; p < W * H; ++p) {
            PCG32Sampler sm;
            sm.seed((uint64_t)p, 1u);
            cam_rays.push_back(camera.pixel_ray(p % W, p / W, sm));
            samplers.push_back(sm);
        }
        std::vector<PrincipalSpectrum> Ls(cam_rays.size());
        std::vector<double> xyz(3 * cam_rays.size());
        if (!integrator.Li(cam_rays.data(), (uint32_t)cam_rays.size(), scene, samplers.data(), Ls.data(), 0,
                           xyz.data())) {
            std::fprintf(stderr, "Li: %s\n", integrator.last_error().c_str());
            rc = 1;
        }
        std::fwrite(xyz.data(), sizeof(double), xyz.size(), out);
        // ... and one ray at a time for the first pixels (the reference's per-ray call)
        for (int p = 0; p < 16 && p < W * H; ++p) {
            PCG32Sampler sm;
            sm.seed((uint64_t)p, 1u);
            const Ray ray = camera.pixel_ray(p % W, p / W, sm);
            double one[3] = {0, 0, 0};
            const PrincipalSpectrum L = integrator.Li(ray, scene, sm, 0, one);
            std::fwrite(one, sizeof(double), 3, out);
            const int same_spectrum = std::memcmp(L.c, Ls[p].c, sizeof(L.c)) == 0;
            const uint64_t rec2[2] = {sm.state, (uint64_t)same_spectrum};
            std::fwrite(rec2, sizeof(uint64_t), 2, out);
        }
        std::fclose(out);
    }
    return rc;
}
