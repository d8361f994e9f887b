/*
 * Out-of-line members of the reference's BVH class (declared in src/filianore/bvh/bvh.h:21-47)
 * implemented on the oracle's CPU BVH, in place of the embree-backed src/filianore/bvh/bvh.cpp.
 *
 * The hit record follows BVH::intersect (bvh.cpp:49-84): t, p = ray.point_at_t(t),
 * pError = abs(p) * gamma<int>(5) (which is 0), n = normalize(Ng), and ray.tMax shrinks.
 * Two fields the reference leaves unset are filled in, without which it cannot render:
 *  - isect->primitive, from a geomID -> Primitive table the harness registers;
 *  - Shading.n = n (the reference's constructor call leaves it NaN);
 *  - uv, from the triangle's vertex uvs and the hit's barycentrics (b1, b2) as
 *    uv0 (1 - b1 - b2) + uv1 b1 + uv2 b2, when the harness registers uvs (it stays (0, 0)
 *    otherwise, as BVH::intersect leaves it);
 *  - dpdu, dpdv (and Shading.dpdu, Shading.dpdv) as Triangle::intersect computes them
 *    (shapes/triangle.cpp:33-52) from the vertex uvs (all zero without uvs). Only the bump
 *    map reads them.
 * Ng = cross(v1 - v0, v2 - v0), the orientation Triangle::sample uses (triangle.cpp:146),
 * so one-sided area lights face the same way for NEE and for BSDF hits.
 * Test infrastructure only.
 */
#include "filianore/bvh/bvh.h"
#include "filianore/core/interaction.h"
#include "filianore/maths/mathutils.h"
#include "../oracle.h"

#include <vector>

namespace ref_shim {
std::vector<const filianore::Primitive *> g_primitives;
std::vector<float> g_uvs;  // 6 per triangle, or empty
}

void rtcReleaseScene(RTCScene scene) {
    if (!scene) return;
    orc_bvh_free(static_cast<orc_bvh *>(scene->accel));
    delete scene;
}

namespace filianore {

void BVH::initialize_scene_geometry(const SceneGeometry &sceneGeometry) {
    bool any = false;
    for (const auto &mesh : sceneGeometry.triangleMeshes) {
        for (const auto &tri : mesh->triangles) {
            add_triangle_mesh(tri);
            any = true;
        }
    }
    if (any) finalise();
}

void BVH::add_triangle_mesh(const std::shared_ptr<BasicTriangle> &tri) {
    const Vector3f *vs[3] = {&tri->v1, &tri->v2, &tri->v3};
    for (const Vector3f *v : vs) {
        scene->verts.push_back(v->x);
        scene->verts.push_back(v->y);
        scene->verts.push_back(v->z);
    }
}

void BVH::finalise() {
    scene->accel = orc_bvh_build(scene->verts.data(), (uint32_t)(scene->verts.size() / 9));
}

bool BVH::intersect(const Ray &ray, SurfaceInteraction *isect) const {
    if (!scene->accel) return false;
    float ot[4] = {ray.origin.x, ray.origin.y, ray.origin.z, ray.tMin};
    float dt[4] = {ray.dir.x, ray.dir.y, ray.dir.z, ray.tMax};
    orc_ray r;
    orc_ray_precompute(ot, dt, &r);
    float t, u, v;
    int32_t id = orc_bvh_closest(static_cast<const orc_bvh *>(scene->accel), &r, &t, &u, &v, nullptr, nullptr);
    if (id < 0) return false;

    *isect = SurfaceInteraction(0, Vector3f(), Vector2f(), Vector3f(), Vector3f(), Vector3f(), Vector3f(),
                                -ray.dir, NULL, 0);
    isect->t = t;
    isect->p = ray.point_at_t(isect->t);
    isect->pError = abs(isect->p) * gamma<int>(5);
    const float *tv = scene->verts.data() + 9 * (size_t)id;
    Vector3f v0(tv[0], tv[1], tv[2]), v1(tv[3], tv[4], tv[5]), v2(tv[6], tv[7], tv[8]);
    isect->n = normalize(cross(v1 - v0, v2 - v0));
    isect->Shading.n = isect->n;
    {
        float q[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (!ref_shim::g_uvs.empty())
            for (int k = 0; k < 6; ++k) q[k] = ref_shim::g_uvs[6 * (size_t)id + k];
        const Vector2f duv02 = Vector2f(q[0], q[1]) - Vector2f(q[4], q[5]);
        const Vector2f duv12 = Vector2f(q[2], q[3]) - Vector2f(q[4], q[5]);
        const Vector3f dp02 = v0 - v2, dp12 = v1 - v2;
        const float determinant = duv02.x * duv12.y - duv02.y * duv12.x;
        const bool degenerate = std::abs(determinant) < 1e-8;
        Vector3f dpdu(0.f), dpdv(0.f);
        if (!degenerate) {
            const float invDet = 1.f / determinant;
            dpdu = (dp02 * duv12.y - dp12 * duv02.y) * invDet;
            dpdv = (dp02 * -duv12.x + dp12 * duv02.x) * invDet;
        }
        if (degenerate || cross(dpdu, dpdv).length_squared() == 0)
            coordinate_system(cross(v1 - v0, v2 - v0), &dpdu, &dpdv);
        isect->dpdu = isect->Shading.dpdu = dpdu;
        isect->dpdv = isect->Shading.dpdv = dpdv;
    }
    isect->primitive = ref_shim::g_primitives[id];
    if (!ref_shim::g_uvs.empty()) {
        const float *q = ref_shim::g_uvs.data() + 6 * (size_t)id;
        const float w = 1.f - u - v;
        isect->uv = Vector2f(q[0] * w + q[2] * u + q[4] * v, q[1] * w + q[3] * u + q[5] * v);
    }
    ray.tMax = isect->t;
    return true;
}

bool BVH::intersect_p(const Ray &ray) const { return false; }

} // namespace filianore
