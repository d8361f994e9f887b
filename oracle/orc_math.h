/*
 * ORACLE — test infrastructure only. Nothing in the product links this file.
 *
 * Float vector arithmetic restated from the reference with the same operation order,
 * so that a build without FMA contraction (-ffp-contract=off) reproduces the
 * reference's results bit for bit:
 *   Vector3 ops             src/filianore/maths/geometry.h:85-163
 *   dot/abs_dot/normalize   src/filianore/maths/geometry.h:202-226
 *   cross (in double)       src/filianore/maths/geometry.h:212-218
 *   coordinate_system       src/filianore/maths/geometry.h:246-256
 *   next_float_up/down      src/filianore/maths/mathutils.h:97-124
 */
#ifndef ORC_MATH_H
#define ORC_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846f
#define ORC_INV_PI 0.31830988618379067154f
#define ORC_INV_2_PI 0.15915494309189533577f
#define ORC_INV_4_PI 0.07957747154594766788f
#define ORC_PI_OVER_2 1.57079632679489661923f
#define ORC_PI_OVER_4 0.78539816339744830961f
#define ORC_SHADOW_EPSILON 0.0001f

typedef struct { float x, y, z; } v3;
typedef struct { float x, y; } v2;

static inline v3 v3m(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 v3_add(v3 a, v3 b) { return v3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 v3_sub(v3 a, v3 b) { return v3m(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 v3_neg(v3 a) { return v3m(-a.x, -a.y, -a.z); }
/* Vector3::operator*(U s) -> (s*x, s*y, s*z) */
static inline v3 v3_mul(v3 a, float s) { return v3m(s * a.x, s * a.y, s * a.z); }
/* Vector3::operator/(U f): multiply by the reciprocal */
static inline v3 v3_div(v3 a, float f) {
    float inv = 1.f / f;
    return v3m(a.x * inv, a.y * inv, a.z * inv);
}
static inline float v3_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float v3_absdot(v3 a, v3 b) { return fabsf(v3_dot(a, b)); }
static inline v3 v3_abs(v3 a) { return v3m(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static inline v3 v3_cross(v3 a, v3 b) {
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
    return v3m((float)((ay * bz) - (az * by)), (float)((az * bx) - (ax * bz)), (float)((ax * by) - (ay * bx)));
}
static inline float v3_len2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline float v3_len(v3 a) { return sqrtf(v3_len2(a)); }
static inline v3 v3_norm(v3 a) { return v3_div(a, v3_len(a)); }
static inline float v3_get(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline void v3_set(v3 *a, int i, float v) {
    if (i == 0) a->x = v; else if (i == 1) a->y = v; else a->z = v;
}

static inline void orc_coordinate_system(v3 v1, v3 *v2, v3 *v3o) {
    if (fabsf(v1.x) > fabsf(v1.y)) {
        float invLen = 1.f / sqrtf(v1.x * v1.x + v1.z * v1.z);
        *v2 = v3m(v1.z * invLen, 0.f, -v1.x * invLen);
    } else {
        float invLen = 1.f / sqrtf(v1.y * v1.y + v1.z * v1.z);
        *v2 = v3m(0.f, v1.z * invLen, -v1.y * invLen);
    }
    *v3o = v3_cross(v1, *v2);
}

static inline uint32_t orc_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float orc_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

static inline float orc_next_float_up(float v) {
    if (isinf(v) && v > 0.f) return v;
    if (v == -0.f) v = 0.f;
    uint32_t ui = orc_f2u(v);
    if (v >= 0) ++ui; else --ui;
    return orc_u2f(ui);
}
static inline float orc_next_float_down(float v) {
    if (isinf(v) && v < 0.f) return v;
    if (v == 0.f) v = -0.f;
    uint32_t ui = orc_f2u(v);
    if (v > 0) --ui; else ++ui;
    return orc_u2f(ui);
}

/* offset_point_origin, src/filianore/core/interaction.h:11-31 */
static inline v3 orc_offset_point_origin(v3 p, v3 pError, v3 n, v3 w) {
    float d = v3_dot(v3_abs(n), pError);
    v3 offset = v3_mul(n, d);
    if (v3_dot(w, n) < 0) offset = v3_neg(offset);
    v3 po = v3_add(p, offset);
    for (int i = 0; i < 3; ++i) {
        float oi = v3_get(offset, i);
        if (oi > 0) v3_set(&po, i, orc_next_float_up(v3_get(po, i)));
        else if (oi < 0) v3_set(&po, i, orc_next_float_down(v3_get(po, i)));
    }
    return po;
}

#endif
