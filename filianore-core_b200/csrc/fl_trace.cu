// Batch ray queries: the replacement of BVH::intersect / rtcIntersect1
// (src/filianore/bvh/bvh.cpp:49-84) and of the shadow test of
// VisibilityEvaluator::unoccluded (src/filianore/illuminants/illuminant.cpp:40-50).
#include <algorithm>

#include "fl_internal.h"
#include "fl_traverse.cuh"

namespace fl {
namespace {

constexpr int kTraceBlock = 128;

__device__ inline void warp_add_u64(unsigned long long *dst, uint32_t v) {
    unsigned long long x = v;
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(dst, x);
}

// traversal steps a lane takes between the warp's refills of finished lanes
#ifndef FL_TRACE_STEPS
#define FL_TRACE_STEPS 8
#endif
constexpr int kTraceSteps = FL_TRACE_STEPS;
// rays per chunk of a host-memory batch: large enough to fill the GPU, small enough that
// a batch of 2^24 rays overlaps copies and traversal over eight chunks
constexpr uint32_t kHostChunk = 1u << 21;

template <int KIND>
struct TraceItem {
    const float4 *org, *dir;
    int4 *hits;
    uint8_t *occ;
    const int32_t *tri_light;
    const WideNode *nodes;
    uint32_t n_nodes;
    const float4 *tris;
    uint32_t n_tris;
    bool any_hit;
    uint32_t q;
    RayPre ray;
    TravState st;
    __device__ bool begin(uint32_t qq) {
        q = qq;
        ray = ray_precompute(__ldg(org + q), __ldg(dir + q));
        trav_init(st, ray);
        return true;
    }
    __device__ void finish() {
        const TraceResult &res = st.res;
        if (KIND == kTraceOccluded) {
            // occluded unless nothing is hit or the closest hit carries an area light
            occ[q] = (res.id >= 0 && (any_hit || (uint32_t)res.id >= n_tris || tri_light[res.id] < 0)) ? 1 : 0;
        } else if (KIND == kTraceClosest) {
            int4 h;
            h.x = res.id;
            h.y = __float_as_int(res.t);
            h.z = __float_as_int(res.id >= 0 ? res.u : 0.f);
            h.w = __float_as_int(res.id >= 0 ? res.v : 0.f);
            hits[q] = h;
        }
    }
};

// persistent kernel: warps refill finished lanes with new rays (fl_traverse.cuh). Compiled for
// 10 resident blocks per SM (at most 48 registers): the ray-cast is latency-bound, and the
// extra warps took the 8.4 M-triangle soup from 599 to 1015 Mrays/s (incoherent) and from
// 1251 to 1805 (coherent) against the compiler's own choice (64 registers, 8 blocks), A/B on
// one B200.
#ifndef FL_TRACE_MIN_BLOCKS
#define FL_TRACE_MIN_BLOCKS 10
#endif
template <int KIND>
__global__ void __launch_bounds__(kTraceBlock, FL_TRACE_MIN_BLOCKS) k_trace(const WideNode *__restrict__ nodes, uint32_t n_nodes,
                                                       const float4 *__restrict__ tris, uint32_t n_tris,
                                                       const int32_t *__restrict__ tri_light, int any_hit_ok,
                                                       const float4 *__restrict__ org, const float4 *__restrict__ dir,
                                                       uint32_t n, int4 *__restrict__ hits, uint8_t *__restrict__ occ,
                                                       int *__restrict__ err, unsigned long long *__restrict__ counters,
                                                       unsigned long long *__restrict__ fetch_counter) {
    TraceItem<KIND> it;
    it.org = org;
    it.dir = dir;
    it.hits = hits;
    it.occ = occ;
    it.tri_light = tri_light;
    it.nodes = nodes;
    it.n_nodes = n_nodes;
    it.tris = tris;
    it.n_tris = n_tris;
    it.any_hit = KIND == kTraceOccluded && any_hit_ok;
    TraceStats st;
    bool error = false;
    uint32_t *fetch = reinterpret_cast<uint32_t *>(fetch_counter);
    __shared__ uint2 stack[trav_stack_smem_bytes(kTraceBlock) / sizeof(uint2)];
    __shared__ uint4 top[kSmemNodeWords];
    const uint32_t n_top = trav_stage_top(top, nodes, n_nodes);
    persistent_trace<kTraceSteps, KIND == kTraceCount>(it, fetch, n, error, st, stack, top, n_top);
    if (KIND == kTraceCount) {
        warp_add_u64(&counters[0], st.nodes);
        warp_add_u64(&counters[1], st.tris);
    }
    if (error) atomicAdd(err, 1);
}

}  // namespace

fl_status launch_trace(Scene *s, const float4 *org, const float4 *dir, uint32_t n, fl_hit *hits, uint8_t *occluded,
                       int kind, cudaStream_t stream, int fetch_slot) {
    if (n == 0) return FL_OK;
    // persistent grid: up to 16 blocks of 128 threads per SM, never more than the rays need
    const uint32_t grid = std::min<uint32_t>((n + kTraceBlock - 1) / kTraceBlock, (uint32_t)s->ctx->sm_count * 16u);
    // the work counter of this launch (launches in flight on different streams use different ones)
    unsigned long long *counters = s->ctx->d_counters + fetch_slot;
    FL_CUDA_TRY(s->ctx, cudaMemsetAsync(counters + 4, 0, sizeof(unsigned long long), stream));
    const int any_hit_ok = s->n_emissive_tris == 0 ? 1 : 0;
    int4 *h = reinterpret_cast<int4 *>(hits);
    switch (kind) {
    case kTraceClosest:
        k_trace<kTraceClosest><<<grid, kTraceBlock, 0, stream>>>(s->nodes, s->n_nodes, s->tris, s->n_tri, s->tri_light,
                                                                 any_hit_ok, org, dir, n, h, occluded,
                                                                 s->ctx->d_error, s->ctx->d_counters, counters + 4);
        break;
    case kTraceOccluded:
        k_trace<kTraceOccluded><<<grid, kTraceBlock, 0, stream>>>(s->nodes, s->n_nodes, s->tris, s->n_tri, s->tri_light,
                                                                  any_hit_ok, org, dir, n, h, occluded,
                                                                  s->ctx->d_error, s->ctx->d_counters, counters + 4);
        break;
    default:
        k_trace<kTraceCount><<<grid, kTraceBlock, 0, stream>>>(s->nodes, s->n_nodes, s->tris, s->n_tri, s->tri_light,
                                                               any_hit_ok, org, dir, n, h, occluded, s->ctx->d_error,
                                                               s->ctx->d_counters, counters + 4);
        break;
    }
    return cuda_status(s->ctx, cudaGetLastError(), "trace launch");
}

}  // namespace fl

using namespace fl;

namespace {

// Runs one query kind over n rays; host buffers are staged through context scratch in chunks.
fl_status trace_common(fl_scene *scene_h, const float *org_tmin, const float *dir_tmax, uint32_t n, fl_hit *hits,
                       uint8_t *occluded, int32_t memory, void *stream_v, int kind, uint64_t *nodes_out,
                       uint64_t *tris_out) {
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!s) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n == 0) return FL_OK;
    if (!org_tmin || !dir_tmax || (kind == kTraceClosest && !hits) || (kind == kTraceOccluded && !occluded)) {
        set_error(ctx, "null ray or result buffer");
        return FL_ERR_INVALID;
    }
    if (memory != FL_MEM_HOST && memory != FL_MEM_DEVICE) {
        set_error(ctx, "memory must be FL_MEM_HOST or FL_MEM_DEVICE");
        return FL_ERR_INVALID;
    }
    cudaStream_t st = stream_v ? reinterpret_cast<cudaStream_t>(stream_v) : ctx->stream;
    FL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(int), st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_counters, 0, 8 * sizeof(unsigned long long), st));
    fl_status rc = FL_OK;
    if (memory == FL_MEM_DEVICE) {
        rc = launch_trace(s, reinterpret_cast<const float4 *>(org_tmin), reinterpret_cast<const float4 *>(dir_tmax), n,
                          hits, occluded, kind, st, 0);
        if (rc) return rc;
    } else {
        // Host buffers: the batch goes through in chunks on two streams that take turns, so
        // the copies of one chunk overlap the traversal of the other (each stream has its
        // own staging buffers and work counter).
        const uint32_t chunk = std::min<uint32_t>(n, kHostChunk);
        const size_t per_ray = 32 + 16 + 1;
        const size_t half = ((size_t)chunk * per_ray + 255) & ~(size_t)255;
        const int lanes = n > chunk ? 2 : 1;
        void *scratch = nullptr;
        if ((rc = ensure_scratch(ctx, half * lanes, &scratch))) return rc;
        if (lanes > 1 && !ctx->stream2) FL_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
        cudaStream_t ss[2] = {st, lanes > 1 ? ctx->stream2 : st};
        if (lanes > 1) {  // the second stream starts after the work already queued on st
            FL_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, st));
            FL_CUDA_TRY(ctx, cudaStreamWaitEvent(ss[1], ctx->ev_fork, 0));
        }
        uint32_t k = 0;
        for (uint32_t off = 0; off < n; off += chunk, ++k) {
            const int l = (int)(k & 1u) % lanes;
            cudaStream_t q = ss[l];
            char *base = static_cast<char *>(scratch) + half * l;
            float4 *d_org = reinterpret_cast<float4 *>(base);
            float4 *d_dir = d_org + chunk;
            fl_hit *d_hits = reinterpret_cast<fl_hit *>(d_dir + chunk);
            uint8_t *d_occ = reinterpret_cast<uint8_t *>(d_hits + chunk);
            const uint32_t m = std::min(chunk, n - off);
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(d_org, org_tmin + 4 * (size_t)off, 16 * (size_t)m, cudaMemcpyHostToDevice, q));
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(d_dir, dir_tmax + 4 * (size_t)off, 16 * (size_t)m, cudaMemcpyHostToDevice, q));
            if ((rc = launch_trace(s, d_org, d_dir, m, d_hits, d_occ, kind, q, l))) return rc;
            if (kind == kTraceClosest)
                FL_CUDA_TRY(ctx, cudaMemcpyAsync(hits + off, d_hits, 16 * (size_t)m, cudaMemcpyDeviceToHost, q));
            else if (kind == kTraceOccluded)
                FL_CUDA_TRY(ctx, cudaMemcpyAsync(occluded + off, d_occ, m, cudaMemcpyDeviceToHost, q));
        }
        if (lanes > 1) {  // st waits for the second stream's chunks
            FL_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_join, ss[1]));
            FL_CUDA_TRY(ctx, cudaStreamWaitEvent(st, ctx->ev_join, 0));
        }
    }
    int err = 0;
    unsigned long long cnt[2] = {0, 0};
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(&err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, ctx->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (nodes_out) *nodes_out = cnt[0];
    if (tris_out) *tris_out = cnt[1];
    if (err) {
        set_error(ctx, std::to_string(err) + " rays hit the traversal stack or iteration bound");
        return FL_ERR_TRAVERSAL;
    }
    return FL_OK;
}

}  // namespace

extern "C" {

fl_status fl_trace_closest(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n, fl_hit *hits,
                           int32_t memory, void *stream) {
    return trace_common(scene, org_tmin, dir_tmax, n, hits, nullptr, memory, stream, kTraceClosest, nullptr, nullptr);
}

fl_status fl_trace_occluded(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n,
                            uint8_t *occluded, int32_t memory, void *stream) {
    return trace_common(scene, org_tmin, dir_tmax, n, nullptr, occluded, memory, stream, kTraceOccluded, nullptr,
                        nullptr);
}

fl_status fl_trace_count(fl_scene *scene, const float *org_tmin, const float *dir_tmax, uint32_t n, int32_t memory,
                         uint64_t *nodes_visited, uint64_t *tris_tested) {
    return trace_common(scene, org_tmin, dir_tmax, n, nullptr, nullptr, memory, nullptr, kTraceCount, nodes_visited,
                        tris_tested);
}

}  // extern "C"
