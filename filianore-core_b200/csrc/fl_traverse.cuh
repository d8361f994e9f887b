// Traversal of the compressed 8-wide BVH (node format in fl_device.cuh).
//
// One thread per ray. The traversal keeps two "groups": a node group (child_base, hit
// bits 24..31 of internal children in octant-permuted slot order | imask in bits 0..7)
// and a triangle group (tri_base, hit bits 0..23 of leaf triangles). The next internal
// child is always the highest set bit, which visits children roughly front to back;
// remaining siblings go to a per-thread stack. Triangles of a node are tested right
// after the node. Loop iterations and stack depth are bounded; hitting a bound sets
// `error` and ends the ray (the host reports FL_ERR_TRAVERSAL).
//
// Closest-hit semantics equal the CPU oracle's: tmin < t < tmax, ties on t resolve to the
// lower soup index, so the answer is independent of traversal order. Box tests are
// conservative (quantised boxes rounded outwards, far distances scaled by 1 + 2^-20).
#pragma once

#include "fl_device.cuh"

namespace fl {

struct TraceResult {
    int id;
    float t, u, v;
};

struct TraceStats {
    uint32_t nodes = 0;
    uint32_t tris = 0;
};

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int b) { return (w >> (8 * b)) & 0xffu; }

// ANY_HIT: stop at the first hit in (tmin, tmax). COUNT: accumulate visit counts.
template <bool ANY_HIT, bool COUNT>
__device__ __forceinline__ TraceResult traverse(const WideNode *__restrict__ nodes, uint32_t n_nodes,
                                                const float4 *__restrict__ tris, uint32_t n_tris, const RayPre &r,
                                                bool &error, TraceStats &stats) {
    TraceResult res;
    res.id = -1;
    res.t = r.tmax;
    res.u = 0.f;
    res.v = 0.f;
    if (!r.valid) return res;

    const float eps = 1e-18f;
    const float idx = 1.f / (fabsf(r.dx) > eps ? r.dx : copysignf(eps, r.dx));
    const float idy = 1.f / (fabsf(r.dy) > eps ? r.dy : copysignf(eps, r.dy));
    const float idz = 1.f / (fabsf(r.dz) > eps ? r.dz : copysignf(eps, r.dz));
    const uint32_t oct = (r.dx < 0.f ? 1u : 0u) | (r.dy < 0.f ? 2u : 0u) | (r.dz < 0.f ? 4u : 0u);
    const uint32_t oct_inv = 7u - oct;
    const float far_scale = 1.00000095367431640625f;  // 1 + 2^-20

    uint2 stack[kTraversalStack];
    int sp = 0;
    uint2 ng = make_uint2(0u, 0x80000000u);
    uint2 tg = make_uint2(0u, 0u);
    uint32_t iter = 0;

    while (true) {
        if (++iter > kTraversalIterLimit) {
            error = true;
            break;
        }
        if (ng.y > 0x00ffffffu) {
            const uint32_t b = 31u - __clz(ng.y & 0xff000000u);
            ng.y &= ~(1u << b);
            const uint32_t slot = (b - 24u) ^ oct_inv;
            const uint32_t rel = __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            const uint32_t ni = ng.x + rel;
            if (ni >= n_nodes) {  // malformed tree: never read outside the node array
                error = true;
                break;
            }
            if (ng.y > 0x00ffffffu) {
                if (sp < kTraversalStack) stack[sp++] = ng;
                else { error = true; break; }
            }
            const uint4 *np = reinterpret_cast<const uint4 *>(nodes + ni);
            const uint4 w0 = __ldg(np + 0);
            const uint4 w1 = __ldg(np + 1);
            const uint4 w2 = __ldg(np + 2);
            const uint4 w3 = __ldg(np + 3);
            const uint4 w4 = __ldg(np + 4);
            if (COUNT) stats.nodes++;
            const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
            const float sx = __uint_as_float((w0.w & 0xffu) << 23);
            const float sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
            const float sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
            const uint32_t imask = w0.w >> 24;
            const float aix = sx * idx, aiy = sy * idy, aiz = sz * idz;
            const float aox = (px - r.ox) * idx, aoy = (py - r.oy) * idy, aoz = (pz - r.oz) * idz;
            // near/far planes by ray direction sign
            const uint32_t lox0 = idx >= 0.f ? w2.x : w3.z, lox1 = idx >= 0.f ? w2.y : w3.w;
            const uint32_t hix0 = idx >= 0.f ? w3.z : w2.x, hix1 = idx >= 0.f ? w3.w : w2.y;
            const uint32_t loy0 = idy >= 0.f ? w2.z : w4.x, loy1 = idy >= 0.f ? w2.w : w4.y;
            const uint32_t hiy0 = idy >= 0.f ? w4.x : w2.z, hiy1 = idy >= 0.f ? w4.y : w2.w;
            const uint32_t loz0 = idz >= 0.f ? w3.x : w4.z, loz1 = idz >= 0.f ? w3.y : w4.w;
            const uint32_t hiz0 = idz >= 0.f ? w4.z : w3.x, hiz1 = idz >= 0.f ? w4.w : w3.y;
            uint32_t hitmask = 0u;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int bsel = i & 3;
                const uint32_t qlx = byte_of(i < 4 ? lox0 : lox1, bsel), qhx = byte_of(i < 4 ? hix0 : hix1, bsel);
                const uint32_t qly = byte_of(i < 4 ? loy0 : loy1, bsel), qhy = byte_of(i < 4 ? hiy0 : hiy1, bsel);
                const uint32_t qlz = byte_of(i < 4 ? loz0 : loz1, bsel), qhz = byte_of(i < 4 ? hiz0 : hiz1, bsel);
                const float tlx = fmaf((float)qlx, aix, aox), thx = fmaf((float)qhx, aix, aox);
                const float tly = fmaf((float)qly, aiy, aoy), thy = fmaf((float)qhy, aiy, aoy);
                const float tlz = fmaf((float)qlz, aiz, aoz), thz = fmaf((float)qhz, aiz, aoz);
                const float tn = fmaxf(fmaxf(tlx, tly), fmaxf(tlz, r.tmin));
                const float tf = fminf(fminf(thx, thy), fminf(thz, res.t)) * far_scale;
                if (tn <= tf) {
                    const uint32_t meta = byte_of(i < 4 ? w1.z : w1.w, bsel);
                    const uint32_t lo5 = meta & 0x1fu;
                    if (lo5 >= 24u) hitmask |= 1u << (24u + ((lo5 - 24u) ^ oct_inv));
                    else hitmask |= (meta >> 5) << lo5;
                }
            }
            ng = make_uint2(w1.x, (hitmask & 0xff000000u) | imask);
            tg = make_uint2(w1.y, hitmask & 0x00ffffffu);
        }
        while (tg.y) {
            const int b = __ffs(tg.y) - 1;
            tg.y &= tg.y - 1u;
            const uint32_t ti = tg.x + (uint32_t)b;
            if (ti >= n_tris) {
                error = true;
                break;
            }
            const float4 a = __ldg(tris + 3 * (size_t)ti);
            const float4 bb = __ldg(tris + 3 * (size_t)ti + 1);
            const float4 c = __ldg(tris + 3 * (size_t)ti + 2);
            if (COUNT) stats.tris++;
            float t, u, v;
            if (intersect_watertight(r, a, bb, c, t, u, v) && t < r.tmax) {
                const int id = __float_as_int(a.w);
                if (ANY_HIT) {
                    res.id = id; res.t = t; res.u = u; res.v = v;
                    return res;
                }
                if (t < res.t || (t == res.t && id < res.id)) {
                    res.id = id; res.t = t; res.u = u; res.v = v;
                }
            }
        }
        if (error) break;
        if (ng.y <= 0x00ffffffu) {
            if (sp == 0) break;
            ng = stack[--sp];
        }
    }
    return res;
}

}  // namespace fl
