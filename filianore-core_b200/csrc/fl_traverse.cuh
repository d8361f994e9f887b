// Traversal of the compressed 8-wide BVH (node format in fl_device.cuh).
//
// The traversal keeps two "groups": a node group (child_base, hit bits 24..31 of internal
// children in octant-permuted slot order | imask in bits 0..7) and a triangle group
// (tri_base, hit bits 0..23 of leaf triangles). The next internal child is always the
// highest set bit, which visits children roughly front to back; remaining siblings go to
// a per-ray stack. Triangles of a node are tested right after the node. Loop iterations,
// stack depth and node/triangle indices are bounded; hitting a bound sets `error` and ends
// the ray (the host reports FL_ERR_TRAVERSAL).
//
// The traversal is a state machine (TravState + trav_step) so that persistent kernels can
// advance many rays a few steps at a time and refill lanes whose ray finished with a new
// ray: a warp then keeps most lanes busy instead of waiting for its longest ray.
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

// Byte b of w as a float. FL_PRMT_CVT 1: one byte permute builds the float 2^23 + byte
// (exponent 150, the byte as mantissa) and one subtraction of 2^23 leaves the byte exactly,
// with integer and FP32 instructions only; 0: an integer-to-float conversion.
#ifndef FL_PRMT_CVT
#define FL_PRMT_CVT 0
#endif
__device__ __forceinline__ float byte_float(uint32_t w, int b) {
    if (FL_PRMT_CVT) return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | (uint32_t)b)) - 8388608.f;
    return (float)byte_of(w, b);
}

struct TravState {
    uint2 ng, tg;
    int sp;
    uint32_t iter;
    float idx, idy, idz;
    uint32_t oct_inv;
    TraceResult res;
};

__device__ __forceinline__ void trav_init(TravState &s, const RayPre &r) {
    const float eps = 1e-18f;
    s.idx = 1.f / (fabsf(r.dx) > eps ? r.dx : copysignf(eps, r.dx));
    s.idy = 1.f / (fabsf(r.dy) > eps ? r.dy : copysignf(eps, r.dy));
    s.idz = 1.f / (fabsf(r.dz) > eps ? r.dz : copysignf(eps, r.dz));
    const uint32_t oct = (r.dx < 0.f ? 1u : 0u) | (r.dy < 0.f ? 2u : 0u) | (r.dz < 0.f ? 4u : 0u);
    s.oct_inv = 7u - oct;
    s.ng = make_uint2(0u, r.valid ? 0x80000000u : 0u);
    s.tg = make_uint2(0u, 0u);
    s.sp = 0;
    s.iter = 0;
    s.res.id = -1;
    s.res.t = r.tmax;
    s.res.u = 0.f;
    s.res.v = 0.f;
}

// Per-lane traversal stack: the first kSmemStack entries live in shared memory (a column per
// lane: entry k of thread t at sm[k * stride + t], so lanes pushing at the same depth hit
// consecutive words), deeper ones in a local-memory spill array that a typical ray never
// touches. Entries are node groups (internal-child hit bits 24..31 set) or postponed
// triangle groups (hit bits 0..23 only).
#ifndef FL_SMEM_STACK
#define FL_SMEM_STACK 8
#endif
constexpr int kSmemStack = FL_SMEM_STACK;
static_assert(kSmemStack > 0 && kSmemStack < kTraversalStack, "shared part of the traversal stack");
struct TravStack {
    uint2 *sm;         // this lane's column
    uint32_t stride;   // threads per block
    const uint4 *top;  // the first n_top wide nodes (the top of the tree), staged in shared memory
    uint32_t n_top;
    uint2 spill[kTraversalStack - kSmemStack];
    __device__ __forceinline__ void put(int k, uint2 v) {
        if (k < kSmemStack) sm[k * stride] = v;
        else spill[k - kSmemStack] = v;
    }
    __device__ __forceinline__ uint2 get(int k) const { return k < kSmemStack ? sm[k * stride] : spill[k - kSmemStack]; }
};
// shared memory a block of `threads` traversal threads needs for its stacks
constexpr size_t trav_stack_smem_bytes(int threads) { return (size_t)threads * kSmemStack * sizeof(uint2); }
__device__ __forceinline__ void trav_stack_bind(TravStack &st, uint2 *smem) {
    st.sm = smem + threadIdx.x;
    st.stride = blockDim.x;
    st.top = nullptr;
    st.n_top = 0;
}

// The top of the tree in shared memory: the collapse numbers wide nodes level by level, so
// the first kSmemNodes nodes are the root and the levels under it, which every ray visits.
// A block stages them once (all its threads call this, with the same arguments) and reads
// them from there instead of through L1.
#ifndef FL_SMEM_NODES
#define FL_SMEM_NODES 0
#endif
constexpr int kSmemNodes = FL_SMEM_NODES;
constexpr int kSmemNodeWords = kSmemNodes > 0 ? kSmemNodes * 5 : 1;
__device__ __forceinline__ uint32_t trav_stage_top(uint4 *smem_nodes, const WideNode *__restrict__ nodes,
                                                   uint32_t n_nodes) {
    const uint32_t n_top = nodes ? min((uint32_t)kSmemNodes, n_nodes) : 0u;
    const uint4 *src = reinterpret_cast<const uint4 *>(nodes);
    for (uint32_t i = threadIdx.x; i < n_top * 5u; i += blockDim.x) smem_nodes[i] = __ldg(src + i);
    __syncthreads();
    return n_top;
}

// Triangle groups are tested when at least this many lanes of the warp test triangles;
// with fewer, the group is pushed and the lanes keep traversing nodes, so that triangle
// tests run with more lanes active (Ylitie, Karras and Laine, HPG 2017). 0 disables it.
#ifndef FL_POSTPONE_LANES
#define FL_POSTPONE_LANES 0
#endif
constexpr int kPostponeLanes = FL_POSTPONE_LANES;

// One traversal step: visit the next node (if any) and test its triangles, then pop.
// Returns true when the ray is finished (no work left, any-hit found, or a bound hit).
template <bool COUNT>
__device__ __forceinline__ bool trav_step(TravState &s, TravStack &stack, const WideNode *__restrict__ nodes,
                                          uint32_t n_nodes, const float4 *__restrict__ tris, uint32_t n_tris,
                                          const RayPre &r, bool any_hit, bool &error, TraceStats &stats) {
    if (++s.iter > kTraversalIterLimit) {
        error = true;
        return true;
    }
    if (s.ng.y > 0x00ffffffu) {
        const uint32_t b = 31u - __clz(s.ng.y & 0xff000000u);
        s.ng.y &= ~(1u << b);
        const uint32_t slot = (b - 24u) ^ s.oct_inv;
        const uint32_t rel = __popc(s.ng.y & 0xffu & ((1u << slot) - 1u));
        const uint32_t ni = s.ng.x + rel;
        if (ni >= n_nodes) {  // malformed tree: never read outside the node array
            error = true;
            return true;
        }
        if (s.ng.y > 0x00ffffffu) {
            if (s.sp < kTraversalStack) stack.put(s.sp++, s.ng);
            else { error = true; return true; }
        }
        uint4 w0, w1, w2, w3, w4;
        if (kSmemNodes > 0 && ni < stack.n_top) {
            const uint4 *np = stack.top + 5 * ni;
            w0 = np[0], w1 = np[1], w2 = np[2], w3 = np[3], w4 = np[4];
        } else {
            const uint4 *np = reinterpret_cast<const uint4 *>(nodes + ni);
            w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
        }
        if (COUNT) stats.nodes++;
        const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
        const float sx = __uint_as_float((w0.w & 0xffu) << 23);
        const float sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23);
        const float sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23);
        const uint32_t imask = w0.w >> 24;
        const float aix = sx * s.idx, aiy = sy * s.idy, aiz = sz * s.idz;
        const float aox = (px - r.ox) * s.idx, aoy = (py - r.oy) * s.idy, aoz = (pz - r.oz) * s.idz;
        const uint32_t lox0 = s.idx >= 0.f ? w2.x : w3.z, lox1 = s.idx >= 0.f ? w2.y : w3.w;
        const uint32_t hix0 = s.idx >= 0.f ? w3.z : w2.x, hix1 = s.idx >= 0.f ? w3.w : w2.y;
        const uint32_t loy0 = s.idy >= 0.f ? w2.z : w4.x, loy1 = s.idy >= 0.f ? w2.w : w4.y;
        const uint32_t hiy0 = s.idy >= 0.f ? w4.x : w2.z, hiy1 = s.idy >= 0.f ? w4.y : w2.w;
        const uint32_t loz0 = s.idz >= 0.f ? w3.x : w4.z, loz1 = s.idz >= 0.f ? w3.y : w4.w;
        const uint32_t hiz0 = s.idz >= 0.f ? w4.z : w3.x, hiz1 = s.idz >= 0.f ? w4.w : w3.y;
        const float far_scale = 1.00000095367431640625f;  // 1 + 2^-20
        uint32_t hitmask = 0u;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int bsel = i & 3;
            const float qlx = byte_float(i < 4 ? lox0 : lox1, bsel), qhx = byte_float(i < 4 ? hix0 : hix1, bsel);
            const float qly = byte_float(i < 4 ? loy0 : loy1, bsel), qhy = byte_float(i < 4 ? hiy0 : hiy1, bsel);
            const float qlz = byte_float(i < 4 ? loz0 : loz1, bsel), qhz = byte_float(i < 4 ? hiz0 : hiz1, bsel);
            const float tlx = fmaf(qlx, aix, aox), thx = fmaf(qhx, aix, aox);
            const float tly = fmaf(qly, aiy, aoy), thy = fmaf(qhy, aiy, aoy);
            const float tlz = fmaf(qlz, aiz, aoz), thz = fmaf(qhz, aiz, aoz);
            const float tn = fmaxf(fmaxf(tlx, tly), fmaxf(tlz, r.tmin));
            const float tf = fminf(fminf(thx, thy), fminf(thz, s.res.t)) * far_scale;
            if (tn <= tf) {
                const uint32_t meta = byte_of(i < 4 ? w1.z : w1.w, bsel);
                const uint32_t lo5 = meta & 0x1fu;
                if (lo5 >= 24u) hitmask |= 1u << (24u + ((lo5 - 24u) ^ s.oct_inv));
                else hitmask |= (meta >> 5) << lo5;
            }
        }
        s.ng = make_uint2(w1.x, (hitmask & 0xff000000u) | imask);
        s.tg = make_uint2(w1.y, hitmask & 0x00ffffffu);
    }
    while (s.tg.y) {
        if (kPostponeLanes > 0 && __popc(__activemask()) < kPostponeLanes && s.ng.y > 0x00ffffffu &&
            s.sp < kTraversalStack) {
            stack.put(s.sp++, s.tg);  // test these with more lanes after the next nodes
            s.tg.y = 0u;
            break;
        }
        const int b = __ffs(s.tg.y) - 1;
        s.tg.y &= s.tg.y - 1u;
        const uint32_t ti = s.tg.x + (uint32_t)b;
        if (ti >= n_tris) {
            error = true;
            return true;
        }
        const float4 a = __ldg(tris + 3 * (size_t)ti);
        const float4 bb = __ldg(tris + 3 * (size_t)ti + 1);
        const float4 c = __ldg(tris + 3 * (size_t)ti + 2);
        if (COUNT) stats.tris++;
        float t, u, v;
        if (intersect_watertight(r, a, bb, c, t, u, v) && t < r.tmax) {
            const int id = __float_as_int(a.w);
            if (any_hit) {
                s.res.id = id; s.res.t = t; s.res.u = u; s.res.v = v;
                return true;
            }
            if (t < s.res.t || (t == s.res.t && id < s.res.id)) {
                s.res.id = id; s.res.t = t; s.res.u = u; s.res.v = v;
            }
        }
    }
    if (s.ng.y <= 0x00ffffffu) {
        if (s.sp == 0) return true;
        const uint2 e = stack.get(--s.sp);
        if (e.y > 0x00ffffffu) s.ng = e;     // a node group
        else { s.tg = e; s.ng.y = 0u; }      // a postponed triangle group
    }
    return false;
}

// Whole traversal of one ray. ANY_HIT: stop at the first hit in (tmin, tmax).
template <bool ANY_HIT, bool COUNT>
__device__ __forceinline__ TraceResult traverse(const WideNode *__restrict__ nodes, uint32_t n_nodes,
                                                const float4 *__restrict__ tris, uint32_t n_tris, const RayPre &r,
                                                TravStack &stack, bool &error, TraceStats &stats) {
    TravState s;
    trav_init(s, r);
    if (!r.valid || n_nodes == 0) return s.res;
    while (!trav_step<COUNT>(s, stack, nodes, n_nodes, tris, n_tris, r, ANY_HIT, error, stats)) {
    }
    return s.res;
}

// Persistent-warp work loop: every lane holds one item; lanes whose item finished fetch
// the next one (one atomic per warp) every `steps` traversal steps. `Item` provides
// begin(q) -> bool (false: nothing to trace, already finished), finish(), the traversal
// state (st, ray, any_hit) and the acceleration structure it traverses (nodes, n_nodes,
// tris, n_tris), which begin() may choose per item. Call with all 32 lanes of the warp.
// `smem` holds the block's traversal stacks (trav_stack_smem_bytes(blockDim.x)).
// top / n_top: the top of the tree staged by trav_stage_top (n_top 0: none), valid for
// every item the kernel traces (one scene).
template <int STEPS, bool COUNT, class Item>
__device__ __forceinline__ void persistent_trace(Item &it, uint32_t *fetch_counter, uint32_t n, bool &error,
                                                 TraceStats &stats, uint2 *smem, const uint4 *top = nullptr,
                                                 uint32_t n_top = 0) {
    TravStack stack;
    trav_stack_bind(stack, smem);
    stack.top = top;
    stack.n_top = n_top;
    bool has = false;
    bool exhausted = false;
    const int lane = threadIdx.x & 31;
    while (true) {
        const uint32_t need = __ballot_sync(0xffffffffu, !has);
        if (need && !exhausted) {
            uint32_t base = 0;
            const int leader = __ffs(need) - 1;
            if (lane == leader) base = atomicAdd(fetch_counter, (uint32_t)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base >= n) exhausted = true;
            if (!has) {
                const uint32_t q = base + __popc(need & ((1u << lane) - 1u));
                if (q < n) {
                    has = it.begin(q);
                    if (has && (it.n_nodes == 0 || !it.ray.valid)) {
                        it.finish();
                        has = false;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, has)) {
            if (exhausted) break;
            continue;
        }
        if (has) {
#pragma unroll 1
            for (int k = 0; k < STEPS; ++k) {
                if (trav_step<COUNT>(it.st, stack, it.nodes, it.n_nodes, it.tris, it.n_tris, it.ray, it.any_hit, error,
                                     stats)) {
                    it.finish();
                    has = false;
                    break;
                }
            }
        }
    }
}

}  // namespace fl
