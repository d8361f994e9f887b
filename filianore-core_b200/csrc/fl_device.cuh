// Device-side building blocks shared by the BVH build, traversal and render kernels.
//
// Rounding: functions whose results must agree bit for bit with the CPU restatement of
// the reference (the watertight triangle test, ray spawning, the hit record) use explicit
// round-to-nearest intrinsics so that nvcc cannot contract them into FMAs. Everything
// else is free to use FMA.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fl {

// ----------------------------------------------------------------------------- constants
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInv4Pi = 0.07957747154594766788f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.78539816339744830961f;
constexpr float kShadowEpsilon = 0.0001f;  // SHADOW_EPSILON, maths/mathutils.h:20

// ----------------------------------------------------------------------------- BVH8 format
// Compressed 8-wide node (80 bytes, five 16-byte words): child boxes are quantised to 8
// bits per axis in the frame (p, 2^e). Child slot order is chosen at build time so that
// traversal in slot order XOR (7 - ray octant) is roughly front to back.
//   meta[i] == 0                 : empty slot
//   meta[i] = 0b001 << 5 | 24+i  : internal child; its node index is
//                                  child_base + popc(imask & ((1 << i) - 1))
//   meta[i] = unary(k) << 5 | off: leaf of k in 1..3 triangles at tri_base + off
struct alignas(16) WideNode {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;  // exponents biased by 127 (scale = 2^(e-127))
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

// Triangle record in BVH order: three float4 (v0.w carries the soup index as int bits).
constexpr int kTriWords = 3;

constexpr int kTraversalStack = 64;             // node-group stack entries per ray
constexpr uint32_t kTraversalIterLimit = 1u << 22;  // bound on loop iterations per ray

// ----------------------------------------------------------------------------- float3 ops
// Reference operation order (maths/geometry.h): (s*x, s*y, s*z), division by reciprocal.
struct v3 {
    float x, y, z;
};
__host__ __device__ inline v3 mk(float x, float y, float z) { return {x, y, z}; }

#if defined(__CUDA_ARCH__)
#define FL_ADD(a, b) __fadd_rn(a, b)
#define FL_SUB(a, b) __fsub_rn(a, b)
#define FL_MUL(a, b) __fmul_rn(a, b)
#define FL_DIV(a, b) __fdiv_rn(a, b)
#else
#define FL_ADD(a, b) ((a) + (b))
#define FL_SUB(a, b) ((a) - (b))
#define FL_MUL(a, b) ((a) * (b))
#define FL_DIV(a, b) ((a) / (b))
#endif

__host__ __device__ inline v3 add(v3 a, v3 b) { return mk(FL_ADD(a.x, b.x), FL_ADD(a.y, b.y), FL_ADD(a.z, b.z)); }
__host__ __device__ inline v3 sub(v3 a, v3 b) { return mk(FL_SUB(a.x, b.x), FL_SUB(a.y, b.y), FL_SUB(a.z, b.z)); }
__host__ __device__ inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ inline v3 mul(v3 a, float s) { return mk(FL_MUL(s, a.x), FL_MUL(s, a.y), FL_MUL(s, a.z)); }
__host__ __device__ inline float dot(v3 a, v3 b) {
    return FL_ADD(FL_ADD(FL_MUL(a.x, b.x), FL_MUL(a.y, b.y)), FL_MUL(a.z, b.z));
}
__host__ __device__ inline float absdot(v3 a, v3 b) { return fabsf(dot(a, b)); }
__host__ __device__ inline v3 vabs(v3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__host__ __device__ inline float len2(v3 a) { return dot(a, a); }
__host__ __device__ inline float len(v3 a) { return sqrtf(len2(a)); }
__host__ __device__ inline v3 divs(v3 a, float f) {
    float inv = FL_DIV(1.f, f);
    return mk(FL_MUL(a.x, inv), FL_MUL(a.y, inv), FL_MUL(a.z, inv));
}
__host__ __device__ inline v3 normalize(v3 a) { return divs(a, len(a)); }
// cross product evaluated in double (maths/geometry.h:212-218)
__host__ __device__ inline v3 cross(v3 a, v3 b) {
    double ax = a.x, ay = a.y, az = a.z, bx = b.x, by = b.y, bz = b.z;
#if defined(__CUDA_ARCH__)
    return mk((float)__dsub_rn(__dmul_rn(ay, bz), __dmul_rn(az, by)),
              (float)__dsub_rn(__dmul_rn(az, bx), __dmul_rn(ax, bz)),
              (float)__dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx)));
#else
    return mk((float)((ay * bz) - (az * by)), (float)((az * bx) - (ax * bz)), (float)((ax * by) - (ay * bx)));
#endif
}
__host__ __device__ inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

__host__ __device__ inline void coordinate_system(v3 v1, v3 *v2, v3 *v3o) {
    if (fabsf(v1.x) > fabsf(v1.y)) {
        float invLen = FL_DIV(1.f, sqrtf(FL_ADD(FL_MUL(v1.x, v1.x), FL_MUL(v1.z, v1.z))));
        *v2 = mk(FL_MUL(v1.z, invLen), 0.f, FL_MUL(-v1.x, invLen));
    } else {
        float invLen = FL_DIV(1.f, sqrtf(FL_ADD(FL_MUL(v1.y, v1.y), FL_MUL(v1.z, v1.z))));
        *v2 = mk(0.f, FL_MUL(v1.z, invLen), FL_MUL(-v1.y, invLen));
    }
    *v3o = cross(v1, *v2);
}

// ----------------------------------------------------------------------------- PCG32
// O'Neill's PCG-XSH-RR with 64-bit state (the generator of src/ext/pcg32.h:40-163).
constexpr uint64_t kPcgMult = 0x5851f42d4c957f2dULL;

struct Pcg32 {
    uint64_t state, inc;
    __host__ __device__ inline uint32_t next() {
        uint64_t old = state;
        state = old * kPcgMult + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31));
    }
    __host__ __device__ inline float nextf() {
        uint32_t u = (next() >> 9) | 0x3f800000u;
#if defined(__CUDA_ARCH__)
        return __fsub_rn(__uint_as_float(u), 1.0f);
#else
        float f;
        __builtin_memcpy(&f, &u, 4);
        return f - 1.0f;
#endif
    }
    __host__ __device__ inline void seed(uint64_t initstate, uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        next();
        state += initstate;
        next();
    }
    // jump ahead by delta draws (Brown 1994, the method of pcg32.h:142-163)
    __host__ __device__ inline void advance(uint64_t delta) {
        uint64_t cur_mult = kPcgMult, cur_plus = inc, acc_mult = 1u, acc_plus = 0u;
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

// ----------------------------------------------------------------------------- rays
struct RayPre {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    bool valid;
};

__device__ inline RayPre ray_precompute(float4 ot, float4 dt) {
    RayPre r;
    r.ox = ot.x; r.oy = ot.y; r.oz = ot.z; r.tmin = ot.w;
    r.dx = dt.x; r.dy = dt.y; r.dz = dt.z; r.tmax = dt.w;
    float ax = fabsf(dt.x), ay = fabsf(dt.y), az = fabsf(dt.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    float d[3] = {dt.x, dt.y, dt.z};
    if (d[kz] < 0.f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.Sx = __fdiv_rn(d[kx], d[kz]);
    r.Sy = __fdiv_rn(d[ky], d[kz]);
    r.Sz = __fdiv_rn(1.f, d[kz]);
    r.valid = (d[kz] != 0.f) && !isnan(d[kz]);
    return r;
}

__device__ inline float sel3(float a, float b, float c, int k) { return k == 0 ? a : (k == 1 ? b : c); }

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013), double-sided, FP32 with
// an FP64 fallback for exactly-zero edge functions. Returns t and the barycentric weights
// of v1 (u) and v2 (v). Bit-identical to the CPU oracle's orc_intersect_watertight.
__device__ inline bool intersect_watertight(const RayPre &r, float4 a4, float4 b4, float4 c4, float &t_out,
                                            float &u_out, float &v_out) {
    const float Ax0 = __fsub_rn(a4.x, r.ox), Ay0 = __fsub_rn(a4.y, r.oy), Az0 = __fsub_rn(a4.z, r.oz);
    const float Bx0 = __fsub_rn(b4.x, r.ox), By0 = __fsub_rn(b4.y, r.oy), Bz0 = __fsub_rn(b4.z, r.oz);
    const float Cx0 = __fsub_rn(c4.x, r.ox), Cy0 = __fsub_rn(c4.y, r.oy), Cz0 = __fsub_rn(c4.z, r.oz);
    const float Akx = sel3(Ax0, Ay0, Az0, r.kx), Aky = sel3(Ax0, Ay0, Az0, r.ky), Akz = sel3(Ax0, Ay0, Az0, r.kz);
    const float Bkx = sel3(Bx0, By0, Bz0, r.kx), Bky = sel3(Bx0, By0, Bz0, r.ky), Bkz = sel3(Bx0, By0, Bz0, r.kz);
    const float Ckx = sel3(Cx0, Cy0, Cz0, r.kx), Cky = sel3(Cx0, Cy0, Cz0, r.ky), Ckz = sel3(Cx0, Cy0, Cz0, r.kz);
    const float Ax = __fsub_rn(Akx, __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(Aky, __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(Bkx, __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(Bky, __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(Ckx, __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(Cky, __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.f) return false;
    const float Az = __fmul_rn(r.Sz, Akz);
    const float Bz = __fmul_rn(r.Sz, Bkz);
    const float Cz = __fmul_rn(r.Sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float t = __fdiv_rn(T, det);
    if (!(t > r.tmin)) return false;
    t_out = t;
    u_out = __fdiv_rn(V, det);
    v_out = __fdiv_rn(W, det);
    return true;
}

}  // namespace fl
