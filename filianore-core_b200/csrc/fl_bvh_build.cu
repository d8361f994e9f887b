// Device construction of the compressed 8-wide BVH that replaces embree's acceleration
// structure (the reference builds it in BVH::initialize_scene_geometry / finalise,
// src/filianore/bvh/bvh.cpp:7-47, via rtcCommitScene).
//
// Pipeline, all on the device:
//   1. per-triangle bounds, centroid bounds (block reduction + atomics)
//   2. 63-bit Morton codes of the centroids, radix sort (CUB) of (code, triangle)
//   3. binary radix tree over the sorted codes (Karras, HPG 2012), ties broken by index
//   4. bottom-up bounds (one climbing thread per leaf, second arrival merges)
//   5. SAH costs of every way to group each binary subtree into up to 8 child slots
//      (dynamic programme, bottom-up like the bounds)
//   6. level-parallel collapse into 8-wide nodes following the programme's choices;
//      children are placed in the slot matching the ray octant that should visit them
//      first; child boxes are quantised to 8 bits per axis, rounded outwards.
// Triangles are rewritten in leaf order as three float4 (v0.w = soup index).
#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cstring>

#include "fl_internal.h"

namespace fl {
namespace {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr int kMaxLeafTris = 3;

__device__ inline uint32_t float_flip(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ inline float float_unflip(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// 1. triangle bounds, centroid bounds (cbounds[0..5]) and scene bounds (cbounds[6..11]), the
// last two as order-preserving uints for atomicMin/Max
__global__ void k_tri_bounds(const float *__restrict__ soup, uint32_t n, float *__restrict__ box,
                             uint32_t *__restrict__ cbounds) {
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float smin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, smax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *v = soup + 9 * (size_t)i;
        for (int a = 0; a < 3; ++a) {
            float lo = fminf(fminf(v[a], v[3 + a]), v[6 + a]);
            float hi = fmaxf(fmaxf(v[a], v[3 + a]), v[6 + a]);
            box[6 * (size_t)i + a] = lo;
            box[6 * (size_t)i + 3 + a] = hi;
            float c = 0.5f * (lo + hi);
            cmin[a] = fminf(cmin[a], c);
            cmax[a] = fmaxf(cmax[a], c);
            smin[a] = fminf(smin[a], lo);
            smax[a] = fmaxf(smax[a], hi);
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            cmin[a] = fminf(cmin[a], __shfl_xor_sync(0xffffffffu, cmin[a], o));
            cmax[a] = fmaxf(cmax[a], __shfl_xor_sync(0xffffffffu, cmax[a], o));
            smin[a] = fminf(smin[a], __shfl_xor_sync(0xffffffffu, smin[a], o));
            smax[a] = fmaxf(smax[a], __shfl_xor_sync(0xffffffffu, smax[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&cbounds[a], float_flip(cmin[a]));
            atomicMax(&cbounds[3 + a], float_flip(cmax[a]));
            atomicMin(&cbounds[6 + a], float_flip(smin[a]));
            atomicMax(&cbounds[9 + a], float_flip(smax[a]));
        }
    }
}

// the host side of float_flip's order-preserving map
inline float host_float_unflip(uint32_t u) {
    const uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    std::memcpy(&f, &b, sizeof f);
    return f;
}

__device__ inline uint64_t spread3_21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

// 2. Morton codes
__global__ void k_morton(const float *__restrict__ box, uint32_t n, const uint32_t *__restrict__ cbounds,
                         uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        float lo = float_unflip(cbounds[a]), hi = float_unflip(cbounds[3 + a]);
        float c = 0.5f * (box[6 * (size_t)i + a] + box[6 * (size_t)i + 3 + a]);
        float ext = hi - lo;
        float x = ext > 0.f ? (c - lo) / ext : 0.f;
        x = fminf(fmaxf(x, 0.f), 1.f);
        q[a] = min((uint32_t)(x * 2097152.0f), 2097151u);
    }
    keys[i] = spread3_21(q[0]) | (spread3_21(q[1]) << 1) | (spread3_21(q[2]) << 2);
    vals[i] = i;
}

__device__ inline int karras_delta(const uint64_t *__restrict__ keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clzll(a ^ b);
}

// 3. binary radix tree: internal node i in [0, n-2]
__global__ void k_karras(const uint64_t *__restrict__ keys, int n, uint32_t *__restrict__ child,
                         uint2 *__restrict__ range, int *__restrict__ parent_int, int *__restrict__ parent_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (karras_delta(keys, n, i, i + 1) - karras_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = karras_delta(keys, n, i, i - d);
    int lmax = 2;
    while (karras_delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (karras_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = karras_delta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (karras_delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    uint32_t left = (first == gamma) ? ((uint32_t)gamma | kLeafBit) : (uint32_t)gamma;
    uint32_t right = (last == gamma + 1) ? ((uint32_t)(gamma + 1) | kLeafBit) : (uint32_t)(gamma + 1);
    child[2 * i] = left;
    child[2 * i + 1] = right;
    range[i] = make_uint2((uint32_t)first, (uint32_t)last);
    if (left & kLeafBit) parent_leaf[gamma] = i; else parent_int[gamma] = i;
    if (right & kLeafBit) parent_leaf[gamma + 1] = i; else parent_int[gamma + 1] = i;
    if (i == 0) parent_int[0] = -1;
}

// 4. bounds: leaf boxes in sorted order, then climb
__global__ void k_refit(const float *__restrict__ trib, const uint32_t *__restrict__ vals, int n,
                        const uint32_t *__restrict__ child, const int *__restrict__ parent_int,
                        const int *__restrict__ parent_leaf, float *leafbox, float *nodebox, int *flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t t = vals[i];
    for (int k = 0; k < 6; ++k) leafbox[6 * (size_t)i + k] = trib[6 * (size_t)t + k];
    if (n < 2) return;
    int node = parent_leaf[i];
    int guard = 0;
    while (node >= 0 && node < n - 1 && guard++ < n) {
        __threadfence();
        if (atomicAdd(&flags[node], 1) == 0) return;
        float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int c = 0; c < 2; ++c) {
            uint32_t ref = child[2 * node + c];
            if ((ref & kLeafBit) ? (ref & ~kLeafBit) >= (uint32_t)n : ref >= (uint32_t)(n - 1)) return;
            const float *src = (ref & kLeafBit) ? leafbox + 6 * (size_t)(ref & ~kLeafBit) : nodebox + 6 * (size_t)ref;
            for (int a = 0; a < 3; ++a) {
                b[a] = fminf(b[a], __ldcg(src + a));
                b[3 + a] = fmaxf(b[3 + a], __ldcg(src + 3 + a));
            }
        }
        for (int k = 0; k < 6; ++k) __stcg(nodebox + 6 * (size_t)node + k, b[k]);
        node = parent_int[node];
    }
}

// 4b. SAH-optimal grouping of the binary tree into 8-wide nodes (the dynamic programme of
// Ylitie, Karras and Laine, HPG 2017). For binary node n and i in 1..8, C(n, i) is the
// least SAH cost of representing n's subtree with at most i child slots of a wide node:
//   C(n, 1) = min(leaf: A(n) c_tri count (count <= 3), internal: A(n) c_node + D(n, 8))
//   C(n, i) = min(C(n, i - 1), D(n, i)),   D(n, j) = min_k C(left, k) + C(right, j - k)
// A binary leaf (one triangle) costs A c_tri for every i. dec[8 n + i - 1] records the choice:
// for i = 1, 0 = leaf and k > 0 = internal with its 8 slots split k / 8 - k; for i > 1, 0 =
// take C(n, i - 1) and k > 0 = split k / i - k between the children. Costs climb the tree like
// the bounds (second arrival computes).
// Triangle-test cost against a node visit, A/B on one B200: 0.3 -> 0.5 -> 0.8 took the
// 8.4 M-triangle soup from 8.0 to 5.3 to 4.4 triangles per incoherent ray (21.0, 22.0, 22.5
// nodes) and from 599 to 709 Mrays/s (0.5, with 64 registers) and 1157 to 1208 (0.8, with
// 48), the render from 888 to 898 Mrays/s; 1.3 measured 1,230 Mrays/s (4.15 / 22.75).
#ifndef FL_SAH_TRI_COST
#define FL_SAH_TRI_COST 1.3f
#endif
constexpr float kCostNode = 1.0f;             // a wide node visit
constexpr float kCostTri = FL_SAH_TRI_COST;   // a triangle test, relative to a node visit

__device__ inline float half_area6(const float *b) {
    const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_sah_costs(int n, const uint32_t *__restrict__ child, const uint2 *__restrict__ range,
                            const int *__restrict__ parent_int, const int *__restrict__ parent_leaf,
                            const float *__restrict__ leafbox, const float *__restrict__ nodebox, float *cost,
                            uint8_t *dec, int *flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || n < 2) return;
    int node = parent_leaf[i];
    int guard = 0;
    while (node >= 0 && node < n - 1 && guard++ < n) {
        __threadfence();
        if (atomicAdd(&flags[node], 1) == 0) return;
        float cc[2][8];
        for (int c = 0; c < 2; ++c) {
            const uint32_t ref = child[2 * node + c];
            if (ref & kLeafBit) {
                if ((ref & ~kLeafBit) >= (uint32_t)n) return;
                const float a = kCostTri * half_area6(leafbox + 6 * (size_t)(ref & ~kLeafBit));
                for (int k = 0; k < 8; ++k) cc[c][k] = a;
            } else {
                if (ref >= (uint32_t)(n - 1)) return;
                for (int k = 0; k < 8; ++k) cc[c][k] = __ldcg(cost + 8 * (size_t)ref + k);
            }
        }
        // D(node, j) for j = 2..8 and the split that gives it
        float D[9];
        uint8_t split[9];
        for (int j = 2; j <= 8; ++j) {
            D[j] = INFINITY;
            split[j] = 1;
            for (int k = 1; k < j; ++k) {
                const float v = cc[0][k - 1] + cc[1][j - k - 1];
                if (v < D[j]) { D[j] = v; split[j] = (uint8_t)k; }
            }
        }
        const float A = half_area6(nodebox + 6 * (size_t)node);
        const uint2 r = range[node];
        const uint32_t count = r.y - r.x + 1;
        const float c_internal = kCostNode * A + D[8];
        const float c_leaf = count <= (uint32_t)kMaxLeafTris ? kCostTri * A * (float)count : INFINITY;
        float C = c_leaf <= c_internal ? c_leaf : c_internal;
        uint8_t d0 = c_leaf <= c_internal ? 0 : split[8];
        __stcg(cost + 8 * (size_t)node, C);
        __stcg(dec + 8 * (size_t)node, d0);
        for (int j = 2; j <= 8; ++j) {
            uint8_t dj = 0;
            if (D[j] < C) { C = D[j]; dj = split[j]; }
            __stcg(cost + 8 * (size_t)node + j - 1, C);
            __stcg(dec + 8 * (size_t)node + j - 1, dj);
        }
        node = parent_int[node];
    }
}

struct BuildCounters {
    uint32_t node_count;
    uint32_t tri_count;
    uint32_t next_count;
    uint32_t leaf_count;
    uint32_t overflow;  // set when an allocation would exceed a buffer (never expected)
};

__device__ inline const float *ref_box(uint32_t ref, const float *leafbox, const float *nodebox) {
    return (ref & kLeafBit) ? leafbox + 6 * (size_t)(ref & ~kLeafBit) : nodebox + 6 * (size_t)ref;
}
__device__ inline uint32_t ref_count(uint32_t ref, const uint2 *range) {
    if (ref & kLeafBit) return 1;
    uint2 r = range[ref];
    return r.y - r.x + 1;
}
__device__ inline uint32_t ref_first(uint32_t ref, const uint2 *range) {
    return (ref & kLeafBit) ? (ref & ~kLeafBit) : range[ref].x;
}

// 5. collapse one level: frontier item (binary ref, wide node index)
__global__ void k_collapse(const uint2 *__restrict__ frontier, uint32_t n_items, uint2 *__restrict__ next,
                           const uint32_t *__restrict__ child, const uint2 *__restrict__ range,
                           const float *__restrict__ leafbox, const float *__restrict__ nodebox,
                           const uint8_t *__restrict__ dec, const uint32_t *__restrict__ vals,
                           const float *__restrict__ soup, WideNode *__restrict__ nodes, float4 *__restrict__ tris,
                           BuildCounters *cnt, uint32_t cap) {
    uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= n_items) return;
    const uint32_t ref = frontier[item].x;
    const uint32_t widx = frontier[item].y;

    uint32_t c[8];
    int count = 0;
    auto valid = [&](uint32_t r) { return (r & kLeafBit) ? (r & ~kLeafBit) < cap : r + 1 < cap; };
    if (!valid(ref)) {
        atomicOr(&cnt->overflow, 2u);
        return;
    }
    // a child slot is a leaf when it is one triangle or the programme chose a leaf for it
    auto is_leaf = [&](uint32_t r) { return (r & kLeafBit) || dec[8 * (size_t)r] == 0; };
    if (is_leaf(ref)) {
        c[0] = ref;  // the whole tree fits one leaf: a root with a single leaf child
        count = 1;
    } else {
        // expand the programme's choices: (binary node, slots) pairs until each is one slot
        uint32_t st_ref[16];
        uint8_t st_slots[16];
        int sp = 0;
        const uint8_t k0 = dec[8 * (size_t)ref];
        st_ref[sp] = child[2 * ref + 1], st_slots[sp++] = (uint8_t)(8 - k0);
        st_ref[sp] = child[2 * ref], st_slots[sp++] = k0;
        while (sp > 0) {
            const uint32_t m = st_ref[--sp];
            uint8_t i = st_slots[sp];
            if (!valid(m) || count >= 8) {
                atomicOr(&cnt->overflow, 2u);
                return;
            }
            if ((m & kLeafBit) || i <= 1) {
                c[count++] = m;
                continue;
            }
            while (i > 1 && dec[8 * (size_t)m + i - 1] == 0) --i;  // fewer slots were as cheap
            if (i <= 1) {
                c[count++] = m;
                continue;
            }
            const uint8_t k = dec[8 * (size_t)m + i - 1];
            if (sp + 2 > 16 || k == 0 || k >= i) {
                atomicOr(&cnt->overflow, 2u);
                return;
            }
            st_ref[sp] = child[2 * m + 1], st_slots[sp++] = (uint8_t)(i - k);
            st_ref[sp] = child[2 * m], st_slots[sp++] = k;
        }
    }

    // node box and child centroids
    float nb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    float cb[8][6];
    for (int k = 0; k < count; ++k) {
        const float *b = ref_box(c[k], leafbox, nodebox);
        for (int a = 0; a < 6; ++a) cb[k][a] = b[a];
        for (int a = 0; a < 3; ++a) {
            nb[a] = fminf(nb[a], b[a]);
            nb[3 + a] = fmaxf(nb[3 + a], b[3 + a]);
        }
    }
    // slot assignment: slot s is visited first by rays whose direction octant is s
    int slot_of[8];
    {
        float nc[3] = {0.5f * (nb[0] + nb[3]), 0.5f * (nb[1] + nb[4]), 0.5f * (nb[2] + nb[5])};
        float cost[8][8];
        for (int k = 0; k < count; ++k) {
            float d[3] = {0.5f * (cb[k][0] + cb[k][3]) - nc[0], 0.5f * (cb[k][1] + cb[k][4]) - nc[1],
                          0.5f * (cb[k][2] + cb[k][5]) - nc[2]};
            for (int s = 0; s < 8; ++s)
                cost[k][s] = ((s & 1) ? -d[0] : d[0]) + ((s & 2) ? -d[1] : d[1]) + ((s & 4) ? -d[2] : d[2]);
        }
        uint32_t used_slots = 0, used_kids = 0;
        for (int it = 0; it < count; ++it) {
            float best = FLT_MAX;
            int bk = -1, bs = -1;
            for (int k = 0; k < count; ++k) {
                if (used_kids & (1u << k)) continue;
                for (int s = 0; s < 8; ++s) {
                    if (used_slots & (1u << s)) continue;
                    if (cost[k][s] < best || bk < 0) { best = cost[k][s]; bk = k; bs = s; }
                }
            }
            used_kids |= 1u << bk;
            used_slots |= 1u << bs;
            slot_of[bk] = bs;
        }
    }
    int kid_in_slot[8];
    for (int s = 0; s < 8; ++s) kid_in_slot[s] = -1;
    for (int k = 0; k < count; ++k) kid_in_slot[slot_of[k]] = k;

    uint32_t n_inner = 0, n_leaf_tris = 0, n_leaves = 0;
    for (int k = 0; k < count; ++k) {
        if (!is_leaf(c[k])) ++n_inner;
        else { n_leaf_tris += ref_count(c[k], range); ++n_leaves; }
    }
    uint32_t child_base = n_inner ? atomicAdd(&cnt->node_count, n_inner) : 0;
    uint32_t tri_base = n_leaf_tris ? atomicAdd(&cnt->tri_count, n_leaf_tris) : 0;
    uint32_t next_base = n_inner ? atomicAdd(&cnt->next_count, n_inner) : 0;
    if (n_leaves) atomicAdd(&cnt->leaf_count, n_leaves);
    // every buffer (nodes, triangles, frontier) holds `cap` = triangle-count entries
    if (widx >= cap || child_base + n_inner > cap || tri_base + n_leaf_tris > cap || next_base + n_inner > cap) {
        atomicOr(&cnt->overflow, 1u);
        return;
    }

    WideNode nd;
    float scale_inv[3];
    uint8_t e8[3];
    for (int a = 0; a < 3; ++a) {
        float ext = __fsub_ru(nb[3 + a], nb[a]);
        float s = __fdiv_ru(ext, 255.f);
        uint32_t bits = __float_as_uint(s);
        int e = (int)((bits >> 23) & 0xff);
        if (bits & 0x7fffff) ++e;
        e = max(1, min(e, 253));
        e8[a] = (uint8_t)e;
        scale_inv[a] = __uint_as_float((uint32_t)(254 - e) << 23);
    }
    nd.px = nb[0]; nd.py = nb[1]; nd.pz = nb[2];
    nd.ex = e8[0]; nd.ey = e8[1]; nd.ez = e8[2];
    nd.child_base = child_base;
    nd.tri_base = tri_base;
    uint8_t imask = 0;
    uint32_t inner_rank = 0, tri_off = 0;
    float p[3] = {nb[0], nb[1], nb[2]};
    for (int s = 0; s < 8; ++s) {
        int k = kid_in_slot[s];
        if (k < 0) {
            nd.meta[s] = 0;
            nd.qlox[s] = nd.qloy[s] = nd.qloz[s] = 0xff;
            nd.qhix[s] = nd.qhiy[s] = nd.qhiz[s] = 0;
            continue;
        }
        uint8_t qlo[3], qhi[3];
        for (int a = 0; a < 3; ++a) {
            float lo = floorf(__fmul_rd(__fsub_rd(cb[k][a], p[a]), scale_inv[a]));
            float hi = ceilf(__fmul_ru(__fsub_ru(cb[k][3 + a], p[a]), scale_inv[a]));
            qlo[a] = (uint8_t)fminf(fmaxf(lo, 0.f), 255.f);
            qhi[a] = (uint8_t)fminf(fmaxf(hi, 0.f), 255.f);
        }
        nd.qlox[s] = qlo[0]; nd.qloy[s] = qlo[1]; nd.qloz[s] = qlo[2];
        nd.qhix[s] = qhi[0]; nd.qhiy[s] = qhi[1]; nd.qhiz[s] = qhi[2];
        uint32_t m = ref_count(c[k], range);
        if (!is_leaf(c[k])) {
            imask |= (uint8_t)(1u << s);
            nd.meta[s] = (uint8_t)((1u << 5) | (24u + (uint32_t)s));
            next[next_base + inner_rank] = make_uint2(c[k], child_base + inner_rank);
            ++inner_rank;
        } else {
            uint32_t unary = (1u << m) - 1u;
            nd.meta[s] = (uint8_t)((unary << 5) | tri_off);
            uint32_t first = ref_first(c[k], range);
            for (uint32_t q = 0; q < m; ++q) {
                uint32_t orig = vals[first + q];
                const float *v = soup + 9 * (size_t)orig;
                float4 *dst = tris + 3 * (size_t)(tri_base + tri_off + q);
                dst[0] = make_float4(v[0], v[1], v[2], __int_as_float((int)orig));
                dst[1] = make_float4(v[3], v[4], v[5], 0.f);
                dst[2] = make_float4(v[6], v[7], v[8], 0.f);
            }
            tri_off += m;
        }
    }
    nd.imask = imask;
    nodes[widx] = nd;
}

// build temporaries from the context's pool, returned to it in stream order
struct Tmp {
    Context *ctx;
    std::vector<void *> ptrs;
    explicit Tmp(Context *c) : ctx(c) {}
    ~Tmp() {
        for (void *p : ptrs) dev_free(ctx, p);
    }
    template <typename T>
    fl_status get(T **p, size_t count) {
        fl_status st = dev_alloc_n(ctx, p, count);
        if (st == FL_OK) ptrs.push_back(*p);
        return st;
    }
};

}  // namespace

fl_status build_bvh(Scene *s) {
    Context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const uint32_t n = s->n_tri;
    s->n_nodes = 0;
    s->n_leaves = 0;
    s->max_depth = 0;
    if (n == 0) return FL_OK;
    if (n > 0x3fffffffu) {
        set_error(ctx, "too many triangles for one scene (limit 2^30)");
        return FL_ERR_INVALID;
    }
    cudaEvent_t ev0, ev1;
    FL_CUDA_TRY(ctx, cudaEventCreate(&ev0));
    FL_CUDA_TRY(ctx, cudaEventCreate(&ev1));
    FL_CUDA_TRY(ctx, cudaEventRecord(ev0, st));

    Tmp tmp(ctx);
    fl_status rc;
    float *trib, *leafbox, *nodebox;
    uint32_t *cbounds, *vals_a, *vals_b, *child;
    uint64_t *keys_a, *keys_b;
    uint2 *range, *front_a, *front_b;
    int *parent_int, *parent_leaf, *flags;
    BuildCounters *cnt;
    WideNode *nodes_big;
    const size_t ni = n > 1 ? n - 1 : 1;
    if ((rc = tmp.get(&trib, 6 * (size_t)n)) || (rc = tmp.get(&leafbox, 6 * (size_t)n)) ||
        (rc = tmp.get(&nodebox, 6 * ni)) || (rc = tmp.get(&cbounds, 12)) ||
        (rc = tmp.get(&vals_a, n)) || (rc = tmp.get(&vals_b, n)) || (rc = tmp.get(&child, 2 * ni)) ||
        (rc = tmp.get(&keys_a, n)) || (rc = tmp.get(&keys_b, n)) || (rc = tmp.get(&range, ni)) ||
        (rc = tmp.get(&front_a, n)) || (rc = tmp.get(&front_b, n)) ||
        (rc = tmp.get(&parent_int, ni)) || (rc = tmp.get(&parent_leaf, n)) ||
        (rc = tmp.get(&flags, ni)) || (rc = tmp.get(&cnt, 1)) || (rc = tmp.get(&nodes_big, n)))
        return rc;
    if ((rc = dev_alloc_n(ctx, &s->tris, 3 * (size_t)n))) return rc;

    const int bs = 256;
    const uint32_t grid_n = (n + bs - 1) / bs;
    uint32_t init_bounds[12] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u,
                                0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(cbounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, st));
    uint32_t grid_b = std::min<uint32_t>(grid_n, (uint32_t)ctx->sm_count * 8u);
    k_tri_bounds<<<grid_b, bs, 0, st>>>(s->soup, n, trib, cbounds);
    k_morton<<<grid_n, bs, 0, st>>>(trib, n, cbounds, keys_a, vals_a);

    cub::DoubleBuffer<uint64_t> dkeys(keys_a, keys_b);
    cub::DoubleBuffer<uint32_t> dvals(vals_a, vals_b);
    size_t temp_bytes = 0;
    FL_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, dkeys, dvals, (int)n, 0, 63, st));
    void *temp;
    if ((rc = tmp.get((char **)&temp, temp_bytes))) return rc;
    FL_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(temp, temp_bytes, dkeys, dvals, (int)n, 0, 63, st));
    const uint64_t *keys = dkeys.Current();
    const uint32_t *vals = dvals.Current();

    if (n >= 2) {
        FL_CUDA_TRY(ctx, cudaMemsetAsync(flags, 0, sizeof(int) * ni, st));
        FL_CUDA_TRY(ctx, cudaMemsetAsync(child, 0, sizeof(uint32_t) * 2 * ni, st));
        FL_CUDA_TRY(ctx, cudaMemsetAsync(range, 0, sizeof(uint2) * ni, st));
        FL_CUDA_TRY(ctx, cudaMemsetAsync(parent_int, 0xff, sizeof(int) * ni, st));
        FL_CUDA_TRY(ctx, cudaMemsetAsync(parent_leaf, 0xff, sizeof(int) * n, st));
        k_karras<<<(uint32_t)((ni + bs - 1) / bs), bs, 0, st>>>(keys, (int)n, child, range, parent_int, parent_leaf);
    }
    k_refit<<<grid_n, bs, 0, st>>>(trib, vals, (int)n, child, parent_int, parent_leaf, leafbox, nodebox, flags);
    float *cost = nullptr;
    uint8_t *dec = nullptr;
    if ((rc = tmp.get(&cost, 8 * ni)) || (rc = tmp.get(&dec, 8 * ni))) return rc;
    if (n >= 2) {
        FL_CUDA_TRY(ctx, cudaMemsetAsync(flags, 0, sizeof(int) * ni, st));
        k_sah_costs<<<grid_n, bs, 0, st>>>((int)n, child, range, parent_int, parent_leaf, leafbox, nodebox, cost, dec,
                                           flags);
    }

    // collapse, one launch per wide level
    BuildCounters c0 = {1u, 0u, 0u, 0u, 0u};
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, &c0, sizeof(c0), cudaMemcpyHostToDevice, st));
    uint2 root = make_uint2(n >= 2 ? 0u : (0u | kLeafBit), 0u);
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(front_a, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    uint32_t items = 1, depth = 0;
    BuildCounters hc{};
    while (items > 0) {
        ++depth;
        if (depth > (uint32_t)kTraversalStack) {
            set_error(ctx, "BVH deeper than the traversal stack");
            return FL_ERR_INVALID;
        }
        FL_CUDA_TRY(ctx, cudaMemsetAsync(&cnt->next_count, 0, sizeof(uint32_t), st));
        k_collapse<<<(items + 127) / 128, 128, 0, st>>>(front_a, items, front_b, child, range, leafbox, nodebox, dec,
                                                        vals, s->soup, nodes_big, s->tris, cnt, n);
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(&hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
        FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        FL_CUDA_TRY(ctx, cudaGetLastError());
        if (hc.overflow) {
            set_error(ctx, "BVH build exceeded its buffers");
            return FL_ERR_INVALID;
        }
        items = hc.next_count;
        std::swap(front_a, front_b);
    }
    if (hc.tri_count != n) {
        set_error(ctx, "BVH build lost triangles");
        return FL_ERR_INVALID;
    }
    s->n_nodes = hc.node_count;
    s->n_leaves = hc.leaf_count;
    s->max_depth = depth;
    if ((rc = dev_alloc_n(ctx, &s->nodes, s->n_nodes))) return rc;
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(s->nodes, nodes_big, sizeof(WideNode) * s->n_nodes, cudaMemcpyDeviceToDevice, st));
    uint32_t sb[6];
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(sb, cbounds + 6, sizeof(sb), cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaEventRecord(ev1, st));
    FL_CUDA_TRY(ctx, cudaEventSynchronize(ev1));
    for (int a = 0; a < 3; ++a) {  // the scene's bounds (for guiding's position encoding)
        s->bmin[a] = host_float_unflip(sb[a]);
        s->bmax[a] = host_float_unflip(sb[3 + a]);
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    s->build_ms = ms;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return FL_OK;
}

}  // namespace fl
