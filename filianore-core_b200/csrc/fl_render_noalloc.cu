// fl_render_noalloc: whole-image rendering that allocates nothing during the call.
//
// Who needs it: hosts that are not allowed to allocate device memory at render time, for
// example a renderer embedded in another application whose device memory is pooled and
// budgeted by that application, or a call made from a context where cudaMalloc would
// implicitly synchronise the device and stall unrelated work. Such a caller sets up the
// context and the scene beforehand and then renders repeatedly without any further
// allocation.
//
// How: the wavefront path state lives in one file-scope device array of kNoAllocScratchBytes
// (32 MiB). It is part of the library's device image, so every GPU that loads the library
// keeps it until the process exits. Waves are sized to fit it, so a frame takes more, smaller
// waves than fl_render. The FP64 accumulation film and the RGB film are the caller's device
// buffers. No cudaMalloc, cudaFree, event creation or allocating library routine is called.
//
// The array is shared by every call in the process: its contents are whatever the last call
// left, and everything that must start at zero is cleared at the start of each call. Calls
// whose GPU work overlaps (different host threads or streams rendering at the same time)
// race on it and produce wrong images.
//
// Set-up: host code cannot use the array's name as a device address (on the host it names a
// shadow variable). The first call on each device, with that device current, asks the runtime
// for the array's device address with cudaGetSymbolAddress and keeps it. With CUDA's lazy
// module loading that first call is also when the driver loads the device code holding the
// array, which reserves its 32 MiB and may synchronise the device: make the first call during
// set-up, before any stream capture and before the caller's memory budget is fixed. Later
// calls allocate nothing.
#include <chrono>
#include <mutex>
#include <string>

#include "fl_render.cuh"

namespace fl {
extern template fl_status render_waves<4>(Scene *, const CamDev &, const fl_render_params &, double *,
                                          WaveCounters *, RenderProfile *, cudaStream_t, void *, size_t,
                                          const LiRays *);
extern template fl_status render_waves<60>(Scene *, const CamDev &, const fl_render_params &, double *,
                                           WaveCounters *, RenderProfile *, cudaStream_t, void *, size_t,
                                           const LiRays *);
CamDev camera_basis_of(const fl_camera &c);

namespace {
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {};
}  // namespace
}  // namespace fl

using namespace fl;

extern "C" fl_status fl_render_noalloc(fl_scene *scene_h, const fl_camera *camera, const fl_render_params *params,
                                       float *film_rgb, double *film_xyz64, fl_render_stats *stats) {
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!s) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!camera || !params || !film_rgb || !film_xyz64) {
        set_error(ctx, "fl_render_noalloc needs a camera, parameters and two device films");
        return FL_ERR_INVALID;
    }
    const fl_render_params p = *params;
    if (!camera_ok(*camera) || p.spp <= 0 || !depths_ok(p) ||
        (p.spectral_mode != FL_SPECTRAL_HERO4 && p.spectral_mode != FL_SPECTRAL_BINS60) || s->n_lights > 64) {
        set_error(ctx, "invalid render parameters");
        return FL_ERR_INVALID;
    }
    if (ctx->device < 0 || ctx->device >= kMaxDevices) {
        set_error(ctx, "fl_render_noalloc supports device indices 0.." + std::to_string(kMaxDevices - 1));
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> g(g_setup_mu);
        if (!g_scratch_addr[ctx->device]) {
            void *addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_status(ctx, e, "cudaGetSymbolAddress(noalloc scratch)");
            g_scratch_addr[ctx->device] = addr;
        }
        scratch = g_scratch_addr[ctx->device];
    }
    // the smallest wave (128 paths) must fit the fixed buffer
    const int nl = (int)s->n_lights;
    const int NL = p.spectral_mode == FL_SPECTRAL_BINS60 ? 60 : 4;
    const size_t per_slot = wave_bytes_per_slot(NL, nl);
    const size_t fixed_overhead = 64 * 1024;  // counters, job table, wave descriptor, array alignment
    if (per_slot * 128 + fixed_overhead > kNoAllocScratchBytes) {
        set_error(ctx, "scene needs more render state per path than the 32 MiB fixed scratch of fl_render_noalloc holds");
        return FL_ERR_CAPACITY;
    }
    fl_render_params q = p;
    q.wave_paths = (int32_t)std::min<size_t>(p.wave_paths > 0 ? (size_t)p.wave_paths : ((size_t)1 << 30),
                                             (kNoAllocScratchBytes - fixed_overhead) / per_slot);
    q.wave_paths = std::max<int32_t>(128, q.wave_paths & ~127);  // never 0, which would mean "the default"
    q.flags = p.flags & FL_RENDER_COUNT;  // no event timing: events would be allocated
    cudaStream_t st = ctx->stream;
    const CamDev cam = camera_basis_of(*camera);
    const size_t n_pix = (size_t)camera->width * camera->height;
    const auto t0 = std::chrono::steady_clock::now();
    // On an error, wait for the kernels already queued before returning: they may still be
    // writing the shared array, and the next call (from any context on this device) must
    // not overlap them.
    auto fail = [&](fl_status code) {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return code;
    };
    cudaError_t ce = cudaMemsetAsync(film_xyz64, 0, n_pix * 3 * sizeof(double), st);
    if (ce != cudaSuccess) return fail(cuda_status(ctx, ce, "film clear"));
    WaveCounters hc{};
    RenderProfile prof;  // off: records nothing
    fl_status rc = NL == 60 ? render_waves<60>(s, cam, q, film_xyz64, &hc, &prof, st, scratch, kNoAllocScratchBytes)
                            : render_waves<4>(s, cam, q, film_xyz64, &hc, &prof, st, scratch, kNoAllocScratchBytes);
    if (rc) return fail(rc);
    k_resolve<<<(uint32_t)std::min<size_t>((n_pix + 255) / 256, (size_t)ctx->sm_count * 8), 256, 0, st>>>(
        film_xyz64, (uint32_t)n_pix, 1.0 / (double)p.spp, film_rgb);
    if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_status(ctx, ce, "resolve launch"));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (stats) {
        *stats = fl_render_stats{};
        stats->paths = hc.paths;
        stats->rays = hc.rays;
        stats->shadow_rays = hc.shadow_rays;
        stats->bounces = hc.bounces;
        stats->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->traversal_errors = (uint32_t)hc.err;
        stats->launches = prof.launches + 1;
        stats->nodes_visited = hc.nodes;
        stats->tris_tested = hc.tris;
        stats->paths_cut = hc.cut;
    }
    return render_bounds_status(ctx, hc);
}
