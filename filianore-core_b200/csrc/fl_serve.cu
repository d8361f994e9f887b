// Serving loop: continuous batching of render jobs (include/filianore_gpu.h, fl_server_*).
//
// A worker thread owns one GPU stream and a fixed set of wave buffers. Each iteration it
//   1. admits queued jobs in arrival order while their films (and their scene, when it is
//      not resident) fit the memory budget, evicting idle scenes least recently used first
//      (fl_serve_sched.h has the policy); newly needed scenes are handed to a builder thread,
//      which uploads them and builds their BVHs on the context's stream while the worker's
//      waves run, and a job takes part in waves from the first wave after its scene is built;
//   2. plans one wave: the path slots are split over the running jobs whose scenes are
//      ready (by the server's packing policy), each job contributing one contiguous range
//      of its samples, so several scenes' paths run in the same kernels;
//   3. uploads the job table and the wave's sample ranges and replays the wave as a CUDA
//      graph captured once at start-up (the launch sequence never changes; the kernels
//      read what to do from device memory);
//   4. after the wave, resolves the films of jobs that are complete and queues their copies
//      to pinned host buffers; a read-out thread waits for each copy and marks the job done,
//      so the worker goes on with the next wave meanwhile. fl_server_poll / fl_server_wait
//      copy the films out of the pinned buffers.
// Jobs that arrive while others run join at the next wave. Per-sample random streams depend
// only on (pixel, sample index), so a job's image is the same alone and in any mix, up to
// the order of the FP64 film additions.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>

#include "fl_render.cuh"
#include "fl_serve_sched.h"

namespace fl {
CamDev camera_basis_of(const fl_camera &c);

namespace {

struct HostScene {
    std::vector<float> verts;
    std::vector<uint32_t> tri_material;
    std::vector<fl_material> materials;
    std::vector<fl_light> lights;
    std::vector<fl_standard_surface> standard;
    std::vector<float> uvs;
    std::vector<std::vector<uint8_t>> pixels;  // one buffer per image
    std::vector<fl_image> images;              // pointing into pixels
    Scene *dev = nullptr;
    uint64_t bytes = 0;
    bool removed = false;  // fl_server_remove_scene: release once no job uses it
};

struct HostJob {
    uint64_t scene = 0;
    fl_camera cam{};
    fl_render_params params{};
    int slot = -1;
    double *d_film = nullptr;
    float *d_rgb = nullptr;
    float *h_rgb = nullptr;    // pinned host copies of the finished films
    double *h_xyz = nullptr;
    fl_status status = FL_ERR_NOT_READY;
    fl_status fail = FL_OK;  // set when admission could not give the job a film; reported when it completes
    bool bound = false;      // its job table entry points at its (built) scene
    double submit_ms = 0, start_ms = 0, done_ms = 0;
};

// A finished job whose film copies to pinned host memory are in flight.
struct Readback {
    uint64_t job;
    cudaEvent_t done;  // recorded after the copies
    double t0;         // when they were queued
};

// Work for the builder thread, done in order: build a scene, or release an evicted or
// removed one (releases queue behind the builds issued before them, so memory is freed in
// the order the scheduler accounted for it).
struct BuildTask {
    uint64_t scene = 0;       // build this scene
    Scene *release = nullptr; // or destroy this one
};

uint64_t scene_bytes_estimate(uint32_t n_tri, uint32_t n_mat) {
    // nodes (< N/2 x 80 B) + BVH triangles 48 B + soup 36 B + material/light tables 8 B
    return (uint64_t)n_tri * (40 + 48 + 36 + 8) + (uint64_t)n_mat * 300 + (1 << 20);
}

}  // namespace

// Streaming iterations per replay of the server's graph: the worker looks at the counters
// (finished jobs, the descriptor's unstarted paths) after each replay. The descriptor is
// topped up while fewer than kServeLookahead / 2 waves (of wave_paths) of its paths are
// unstarted: fewer keeps a new job's samples closer to the front, more keeps every slot
// busy between two looks.
#ifndef FL_SERVE_ITERS
#define FL_SERVE_ITERS 2
#endif
#ifndef FL_SERVE_LOOKAHEAD
#define FL_SERVE_LOOKAHEAD 4
#endif
constexpr int kServeIters = FL_SERVE_ITERS;
// the trace queues alternate by iteration parity and a replay always starts at parity 0
static_assert(kServeIters > 0 && kServeIters % 2 == 0, "an even number of iterations per replay");
constexpr uint32_t kServeLookahead = FL_SERVE_LOOKAHEAD;

struct Server {
    Context *ctx = nullptr;
    fl_server_config cfg{};
    cudaStream_t stream = nullptr;
    cudaStream_t rstream = nullptr;       // film read-outs
    cudaEvent_t ev_resolved = nullptr;    // a finished film is resolved (read-outs wait on it)
    void *wave_mem = nullptr;
    size_t wave_bytes = 0;
    WaveBuffers W{};
    cudaGraphExec_t graph = nullptr;  // kServeIters streaming iterations
    std::vector<JobDev> table;  // kMaxJobs
    WaveDesc desc{};            // the device descriptor's host copy
    unsigned long long *d_job_done = nullptr;  // finished paths per job table entry
    unsigned long long *h_done = nullptr;      // pinned copies of the counters
    WaveCounters *h_cnt = nullptr;
    std::vector<int> free_slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    int removals = 0;  // scenes removed by the caller and not yet released
    uint64_t events = 0;  // submissions, removals and finished builds: the worker looks again
    std::thread worker;
    std::thread builder;
    std::deque<BuildTask> build_q;
    std::condition_variable cv_build;
    std::thread reader;
    std::deque<Readback> read_q;
    std::condition_variable cv_read;
    std::vector<cudaEvent_t> free_events;
    // pinned host buffers for finished films, kept by size for the next jobs
    std::multimap<size_t, void *> pinned_pool;
    // FL_SERVE_TRACE=<file>: one line per wave, build and film read-out, appended at destroy
    bool tracing = false;
    std::string trace_path;
    std::vector<std::string> trace;
    void trace_event(const char *kind, double t0, double ms, uint64_t id, uint64_t n) {
        if (!tracing) return;
        char b[160];
        std::snprintf(b, sizeof(b), "%s,%.3f,%.3f,%llu,%llu", kind, t0, ms, (unsigned long long)id,
                      (unsigned long long)n);
        trace.emplace_back(b);
    }
    ServeScheduler sched;
    std::map<uint64_t, HostScene> scenes;
    std::map<uint64_t, std::unique_ptr<HostJob>> jobs;
    uint64_t next_scene = 1, next_job = 1;
    std::chrono::steady_clock::time_point t0;
    fl_server_stats stats{};
    std::string error;
    // Film buffers come from the context's stream-ordered pool on the server's stream:
    // cudaMalloc / cudaFree would synchronise the device and stall the waves per job.
    void *acquire(size_t bytes) {
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, bytes, ctx->pool, stream) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return p;
    }
    void release(void *p, size_t) {
        if (p) cudaFreeAsync(p, stream);
    }
    void *acquire_pinned(size_t bytes) {
        auto it = pinned_pool.find(bytes);
        if (it != pinned_pool.end()) {
            void *p = it->second;
            pinned_pool.erase(it);
            return p;
        }
        void *p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return p;
    }
    void release_pinned(void *p, size_t bytes) {
        if (p) pinned_pool.insert({bytes, p});  // kept until the server is destroyed (cudaFreeHost synchronises)
    }

    Server(uint64_t budget, int max_jobs, int policy) : sched(budget, max_jobs, policy) {
        sched.set_async_builds(true);
    }
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

fl_status make_scene(Server *S, const HostScene &h, Scene **out_scene) {
    fl_scene_desc d{};
    d.verts = h.verts.data();
    d.n_tri = (uint32_t)(h.verts.size() / 9);
    d.tri_material = h.tri_material.data();
    d.materials = h.materials.data();
    d.n_materials = (uint32_t)h.materials.size();
    d.lights = h.lights.data();
    d.n_lights = (uint32_t)h.lights.size();
    d.standard_surfaces = h.standard.empty() ? nullptr : h.standard.data();
    d.n_standard_surfaces = (uint32_t)h.standard.size();
    d.uvs = h.uvs.empty() ? nullptr : h.uvs.data();
    d.images = h.images.empty() ? nullptr : h.images.data();
    d.n_images = (uint32_t)h.images.size();
    fl_scene *out = nullptr;
    fl_status rc = fl_scene_create(reinterpret_cast<fl_context *>(S->ctx), &d, &out);
    *out_scene = rc == FL_OK ? reinterpret_cast<Scene *>(out) : nullptr;
    return rc;
}

// Builds and releases scenes in the order the worker queued them. A scene whose build
// failed is still marked built; its jobs then fail with FL_ERR_OOM when they are bound.
void builder_loop(Server *S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lock(S->mu);
    while (true) {
        S->cv_build.wait(lock, [&] { return S->stop || !S->build_q.empty(); });
        if (S->stop) break;  // fl_server_destroy releases what is left
        const BuildTask t = S->build_q.front();
        S->build_q.pop_front();
        if (t.release) {
            lock.unlock();
            fl_scene_destroy(reinterpret_cast<fl_scene *>(t.release));
            lock.lock();
            continue;
        }
        auto it = S->scenes.find(t.scene);
        if (it == S->scenes.end()) continue;
        // the map node stays: a job that waits for this scene holds it until the scene is built
        const HostScene *h = &it->second;
        Scene *dev = h->dev;
        fl_status rc = FL_OK;
        if (!dev) {
            lock.unlock();
            const double b0 = S->now_ms();
            rc = make_scene(S, *h, &dev);
            const double ms = S->now_ms() - b0;
            lock.lock();
            S->stats.build_ms += ms;
            S->stats.build_max_ms = std::max(S->stats.build_max_ms, ms);
            S->trace_event("build", b0, ms, t.scene, h->verts.size() / 9);
        }
        it->second.dev = dev;
        if (rc == FL_OK) S->stats.builds++;
        S->sched.scene_built(t.scene);
        S->events++;
        S->cv_work.notify_one();
    }
}

// Resolves a finished job's film and queues its copies to pinned host memory; the read-out
// thread completes the job when they have arrived. Called by the worker without the lock.
void finish_job(Server *S, uint64_t jid, HostJob &job) {
    const double t0 = S->now_ms();
    const size_t n_pix = (size_t)job.cam.width * job.cam.height;
    k_resolve<<<(uint32_t)std::min<size_t>((n_pix + 255) / 256, (size_t)S->ctx->sm_count * 8), 256, 0, S->stream>>>(
        job.d_film, (uint32_t)n_pix, 1.0 / (double)job.params.spp, job.d_rgb);
    // the copies run on the read-out stream, after the resolve, while the next waves run
    cudaEvent_t ev = nullptr;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        job.h_rgb = static_cast<float *>(S->acquire_pinned(n_pix * 3 * sizeof(float)));
        job.h_xyz = static_cast<double *>(S->acquire_pinned(n_pix * 3 * sizeof(double)));
        if (!S->free_events.empty()) {
            ev = S->free_events.back();
            S->free_events.pop_back();
        }
    }
    cudaError_t e = job.h_rgb && job.h_xyz ? cudaSuccess : cudaErrorMemoryAllocation;
    if (e == cudaSuccess && !ev) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(S->ev_resolved, S->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S->rstream, S->ev_resolved, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(job.h_rgb, job.d_rgb, n_pix * 3 * sizeof(float), cudaMemcpyDeviceToHost, S->rstream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(job.h_xyz, job.d_film, n_pix * 3 * sizeof(double), cudaMemcpyDeviceToHost, S->rstream);
    if (e == cudaSuccess) e = cudaEventRecord(ev, S->rstream);
    std::lock_guard<std::mutex> lock(S->mu);
    if (job.slot >= 0) S->free_slots.push_back(job.slot);  // no later wave uses its table entry
    job.slot = -1;
    if (e == cudaSuccess) {
        S->read_q.push_back(Readback{jid, ev, t0});
        S->cv_read.notify_one();
    } else {
        cudaGetLastError();
        if (ev) S->free_events.push_back(ev);
        S->release(job.d_film, n_pix * 3 * sizeof(double));
        S->release(job.d_rgb, n_pix * 3 * sizeof(float));
        job.d_film = nullptr;
        job.d_rgb = nullptr;
        job.status = e == cudaErrorMemoryAllocation ? FL_ERR_OOM : FL_ERR_CUDA;
        job.done_ms = S->now_ms();
        S->stats.jobs_done++;
        S->cv_done.notify_all();
    }
    S->stats.finish_ms += S->now_ms() - t0;
}

// Waits for the queued film copies in order and completes their jobs.
void reader_loop(Server *S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lock(S->mu);
    while (true) {
        S->cv_read.wait(lock, [&] { return S->stop || !S->read_q.empty(); });
        if (S->read_q.empty()) break;  // stopping, with nothing in flight
        const Readback r = S->read_q.front();
        S->read_q.pop_front();
        lock.unlock();
        const cudaError_t e = cudaEventSynchronize(r.done);
        lock.lock();
        S->free_events.push_back(r.done);
        HostJob &job = *S->jobs[r.job];
        const size_t n_pix = (size_t)job.cam.width * job.cam.height;
        S->release(job.d_film, n_pix * 3 * sizeof(double));
        S->release(job.d_rgb, n_pix * 3 * sizeof(float));
        job.d_film = nullptr;
        job.d_rgb = nullptr;
        job.status = e == cudaSuccess ? FL_OK : FL_ERR_CUDA;
        job.done_ms = S->now_ms();
        S->stats.jobs_done++;
        S->trace_event("readout", r.t0, job.done_ms - r.t0, r.job, n_pix);
        S->cv_done.notify_all();
    }
}

// Completes the running jobs whose paths have all finished on the device (or that have no
// film: their samples were skipped), in the worker without the lock held.
void complete_jobs(Server *S, const std::vector<uint64_t> &done) {
    for (uint64_t jid : done) {
        HostJob *job;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            job = S->jobs[jid].get();
        }
        if (job->d_film) finish_job(S, jid, *job);
        else {
            std::lock_guard<std::mutex> lock(S->mu);
            job->done_ms = S->now_ms();
            job->status = job->fail != FL_OK ? job->fail : FL_ERR_OOM;
            if (job->slot >= 0) S->free_slots.push_back(job->slot);
            job->slot = -1;
            S->stats.jobs_done++;
        }
    }
    if (!done.empty()) S->cv_done.notify_all();
}

void worker_loop(Server *S) {
    cudaSetDevice(S->ctx->device);
    const size_t desc_head = offsetof(WaveDesc, seg);
    const uint32_t cap = (uint32_t)S->W.cap;
    uint64_t seen = 0;
    bool progressed = true;   // the last iteration ran device work or completed jobs
    bool busy = false;        // paths in flight or not yet started on the device
    WaveCounters &hc = *S->h_cnt;
    while (true) {
        ServeScheduler::Admission adm;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            // with nothing to run (every running job waits for its scene) wait for news
            const auto i0 = std::chrono::steady_clock::now();
            S->cv_work.wait(lock, [&] {
                return S->stop || S->events != seen || (progressed && (busy || !S->sched.idle()));
            });
            S->stats.idle_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - i0).count();
            if (S->stop) break;
            seen = S->events;
            adm = S->sched.admit();
            // scenes: release, then build, in this order on the builder thread
            for (uint64_t sid : adm.evict) {
                HostScene &h = S->scenes[sid];
                if (h.dev) S->build_q.push_back(BuildTask{0, h.dev});
                h.dev = nullptr;
                S->stats.evictions++;
            }
            for (uint64_t sid : adm.build) S->build_q.push_back(BuildTask{sid, nullptr});
            for (uint64_t jid : adm.rejected) {
                auto it = S->jobs.find(jid);
                if (it != S->jobs.end()) it->second->status = FL_ERR_CAPACITY;
            }
        }
        if (!adm.evict.empty() || !adm.build.empty()) S->cv_build.notify_one();
        if (!adm.rejected.empty()) S->cv_done.notify_all();
        std::vector<uint64_t> done;
        bool table_changed = false, desc_changed = false;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            for (uint64_t jid : adm.admitted) {
                HostJob &job = *S->jobs[jid];
                const size_t n_pix = (size_t)job.cam.width * job.cam.height;
                bool ok = !S->free_slots.empty();
                if (ok) job.d_film = static_cast<double *>(S->acquire(n_pix * 3 * sizeof(double)));
                if (ok) job.d_rgb = static_cast<float *>(S->acquire(n_pix * 3 * sizeof(float)));
                if (!job.d_film || !job.d_rgb) ok = false;
                if (!ok) {
                    S->release(job.d_film, n_pix * 3 * sizeof(double));
                    S->release(job.d_rgb, n_pix * 3 * sizeof(float));
                    job.d_rgb = nullptr;
                    job.d_film = nullptr;
                    job.fail = FL_ERR_OOM;  // the scheduler still runs it; its samples are skipped
                    continue;
                }
                cudaMemsetAsync(job.d_film, 0, n_pix * 3 * sizeof(double), S->stream);
                job.slot = S->free_slots.back();
                S->free_slots.pop_back();
            }
            // jobs whose scenes are now built join; a failed build fails its jobs
            for (uint64_t jid : S->sched.running_jobs()) {
                HostJob &job = *S->jobs[jid];
                if (job.bound || job.slot < 0 || !S->sched.scene_ready(job.scene)) continue;
                const HostScene &h = S->scenes[job.scene];
                job.bound = true;
                job.start_ms = S->now_ms();
                if (h.dev) {
                    S->table[job.slot] = job_of(h.dev, camera_basis_of(job.cam), job.params, job.d_film);
                    cudaMemsetAsync(S->d_job_done + job.slot, 0, sizeof(unsigned long long), S->stream);
                    S->h_done[job.slot] = 0;
                    table_changed = true;
                } else {
                    const size_t n_pix = (size_t)job.cam.width * job.cam.height;
                    S->release(job.d_film, n_pix * 3 * sizeof(double));
                    S->release(job.d_rgb, n_pix * 3 * sizeof(float));
                    job.d_film = nullptr;
                    job.d_rgb = nullptr;
                    job.fail = FL_ERR_OOM;
                    S->free_slots.push_back(job.slot);
                    job.slot = -1;
                }
            }
            // Top the descriptor up while fewer than two waves of its paths are unstarted:
            // its unstarted remainder, then the scheduler's next plan of samples.
            const uint32_t started = busy ? hc.next_path : S->desc.n_wave;
            const uint32_t unstarted = S->desc.n_wave - std::min(started, S->desc.n_wave);
            const uint32_t ahead = (uint32_t)(((uint64_t)cap * kServeLookahead) / 2);
            if (unstarted < ahead) {
                WaveDesc nd{};
                uint32_t pos = 0;
                for (uint32_t k = 0; k < S->desc.n_seg; ++k) {  // the remainder
                    const WaveSeg &sg = S->desc.seg[k];
                    const uint32_t b = std::max(sg.slot_begin, started), e = sg.slot_begin + sg.count;
                    if (b >= e) continue;
                    nd.seg[nd.n_seg++] = WaveSeg{sg.job, pos, e - b, 0u, sg.sample_base + (b - sg.slot_begin), 0ull};
                    pos += e - b;
                }
                // a plan adds at most one range per running job
                if (nd.n_seg + (uint32_t)S->sched.running() <= (uint32_t)kMaxSegs) {
                    for (const auto &sg : S->sched.plan_wave(ahead - unstarted)) {
                        HostJob &job = *S->jobs[sg.job];
                        S->stats.paths += sg.count;
                        if (job.slot < 0) continue;  // failed admission: its samples are skipped
                        WaveSeg *last = nd.n_seg ? &nd.seg[nd.n_seg - 1] : nullptr;
                        if (last && last->job == (uint32_t)job.slot &&
                            last->sample_base + last->count == sg.sample_base)
                            last->count += sg.count;  // the same job's next samples
                        else
                            nd.seg[nd.n_seg++] = WaveSeg{(uint32_t)job.slot, pos, sg.count, 0u, sg.sample_base, 0ull};
                        pos += sg.count;
                    }
                    S->stats.waves++;
                }
                nd.n_wave = pos;
                if (pos > unstarted) {  // new samples: the device goes on with nd from its start
                    S->desc = nd;
                    desc_changed = true;
                }
            }
            // jobs without a film whose samples are all dispatched complete now
            for (uint64_t jid : S->sched.running_jobs()) {
                const HostJob &job = *S->jobs[jid];
                if (job.slot < 0 && S->sched.dispatched_all(jid)) done.push_back(jid);
            }
            for (uint64_t jid : done) S->sched.complete(jid);
        }
        if (table_changed)
            cudaMemcpyAsync(S->W.d_jobs, S->table.data(), sizeof(JobDev) * kMaxJobs, cudaMemcpyHostToDevice, S->stream);
        if (desc_changed) {
            cudaMemcpyAsync(S->W.d_wave, &S->desc, desc_head + sizeof(WaveSeg) * S->desc.n_seg, cudaMemcpyHostToDevice,
                            S->stream);
            cudaMemsetAsync(&S->W.A.cnt->next_path, 0, sizeof(uint32_t), S->stream);
            hc.next_path = 0;
        }
        busy = busy || S->desc.n_wave > 0;
        progressed = !done.empty();
        if (busy) {
            // a few iterations, then the counters: live paths, started paths, finished paths per job
            const double w0 = S->now_ms();
            cudaGraphLaunch(S->graph, S->stream);
            cudaMemcpyAsync(S->h_cnt, S->W.A.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, S->stream);
            cudaMemcpyAsync(S->h_done, S->d_job_done, sizeof(unsigned long long) * kMaxJobs, cudaMemcpyDeviceToHost,
                            S->stream);
            const cudaError_t e = cudaStreamSynchronize(S->stream);
            const double ms = S->now_ms() - w0;
            busy = e == cudaSuccess && !(hc.n_next == 0 && hc.next_path >= S->desc.n_wave);
            progressed = true;
            std::vector<uint64_t> fin;
            {
                std::lock_guard<std::mutex> lock(S->mu);
                S->stats.busy_ms += ms;
                S->stats.wave_max_ms = std::max(S->stats.wave_max_ms, ms);
                S->trace_event("iters", w0, ms, hc.n_next, hc.next_path);
                if (e != cudaSuccess) S->error = cudaGetErrorString(e);
                if (hc.err) S->error = "traversal or queue bound hit in a server wave";
                for (uint64_t jid : S->sched.running_jobs()) {
                    const HostJob &job = *S->jobs[jid];
                    if (job.slot < 0 || !job.bound || !S->sched.dispatched_all(jid)) continue;
                    const uint64_t total = (uint64_t)job.cam.width * job.cam.height * (uint64_t)job.params.spp;
                    if (S->h_done[job.slot] >= total || e != cudaSuccess) fin.push_back(jid);
                }
                for (uint64_t jid : fin) S->sched.complete(jid);
            }
            done.insert(done.end(), fin.begin(), fin.end());
        }
        complete_jobs(S, done);
        // scenes removed by the caller that no job uses any more
        bool dropped = false;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            for (auto it = S->scenes.begin(); S->removals > 0 && it != S->scenes.end();) {
                if (it->second.removed && S->sched.scene_unused(it->first)) {
                    S->sched.forget_scene(it->first);
                    S->removals--;
                    if (it->second.dev) {
                        S->build_q.push_back(BuildTask{0, it->second.dev});
                        dropped = true;
                    }
                    it = S->scenes.erase(it);
                } else {
                    ++it;
                }
            }
        }
        if (dropped) S->cv_build.notify_one();
    }
}

}  // namespace
}  // namespace fl

using namespace fl;

extern "C" {

fl_status fl_server_create(fl_context *ctx_h, const fl_server_config *cfg, fl_server **out) {
    Context *ctx = reinterpret_cast<Context *>(ctx_h);
    if (!ctx || !cfg || !out) return FL_ERR_INVALID;
    *out = nullptr;
    if (cfg->memory_budget_bytes == 0 || cfg->max_jobs <= 0 || cfg->max_jobs > kMaxJobs || cfg->max_depth < 0 ||
        cfg->max_depth > 250 || cfg->max_lights < 0 || cfg->max_lights > 64 || cfg->policy < 0 || cfg->policy > 6) {
        set_error(ctx, "invalid server configuration");
        return FL_ERR_INVALID;
    }
    auto S = std::make_unique<Server>(cfg->memory_budget_bytes, cfg->max_jobs, cfg->policy);
    S->ctx = ctx;
    S->cfg = *cfg;
    S->t0 = std::chrono::steady_clock::now();
    if (const char *tp = std::getenv("FL_SERVE_TRACE")) {
        S->tracing = tp[0] != 0;
        S->trace_path = tp;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    // scene memory the budget allows stays cached in the context's pool between builds
    if (ctx->pool) {
        uint64_t cur = 0, keep = std::max<uint64_t>(kPoolKeepBytes, cfg->memory_budget_bytes);
        if (cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && keep > cur)
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    FL_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    cudaError_t es = cudaStreamCreateWithFlags(&S->rstream, cudaStreamNonBlocking);
    if (es == cudaSuccess) es = cudaEventCreateWithFlags(&S->ev_resolved, cudaEventDisableTiming);
    if (es != cudaSuccess) {
        if (S->rstream) cudaStreamDestroy(S->rstream);
        cudaStreamDestroy(S->stream);
        return cuda_status(ctx, es, "server streams");
    }
    auto drop_streams = [&] {
        cudaEventDestroy(S->ev_resolved);
        cudaStreamDestroy(S->rstream);
        cudaStreamDestroy(S->stream);
    };
    const size_t cap = cfg->wave_paths > 0 ? (size_t)cfg->wave_paths : ((size_t)1 << 21);
    const size_t per_slot = wave_bytes_per_slot(4, cfg->max_lights);
    S->wave_bytes = cap * per_slot + (1 << 20);
    cudaError_t e = cudaMalloc(&S->wave_mem, S->wave_bytes);
    if (e != cudaSuccess) {
        drop_streams();
        return cuda_status(ctx, e, "server wave buffers");
    }
    fl_status rc = wave_buffers(ctx, 4, cfg->max_lights, cap, S->wave_mem, S->wave_bytes, S->W);
    if (rc) {
        cudaFree(S->wave_mem);
        drop_streams();
        return rc;
    }
    S->table.assign(kMaxJobs, JobDev{});
    for (int i = cfg->max_jobs - 1; i >= 0; --i) S->free_slots.push_back(i);
    e = cudaMalloc(&S->d_job_done, sizeof(unsigned long long) * kMaxJobs);
    if (e == cudaSuccess) e = cudaHostAlloc(&S->h_done, sizeof(unsigned long long) * kMaxJobs, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&S->h_cnt, sizeof(WaveCounters), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaFree(S->d_job_done);
        cudaFreeHost(S->h_done);
        cudaFree(S->wave_mem);
        drop_streams();
        return cuda_status(ctx, e, "server counters");
    }
    std::memset(S->h_done, 0, sizeof(unsigned long long) * kMaxJobs);
    std::memset(S->h_cnt, 0, sizeof(WaveCounters));
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    // streaming waves: every slot free, an empty descriptor, finished paths counted per job
    S->W.A.slot_free = S->W.slot_free;
    S->W.A.free_count = S->W.free_count;
    S->W.A.free_off = S->W.free_off;
    S->W.A.job_done = S->d_job_done;
    cudaMemsetAsync(S->W.A.cnt, 0, sizeof(WaveCounters), S->stream);
    cudaMemsetAsync(S->W.d_wave, 0, offsetof(WaveDesc, seg), S->stream);
    cudaMemsetAsync(S->d_job_done, 0, sizeof(unsigned long long) * kMaxJobs, S->stream);
    k_stream_init<<<std::min<uint32_t>(((uint32_t)S->W.cap + 127) / 128, (uint32_t)sms * 8), 128, 0, S->stream>>>(S->W.A);
    shade_shapes<4, false>();  // launch shapes, outside the capture
    // capture kServeIters streaming iterations once; the worker replays them
    RenderProfile prof;
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        // the server's waves may carry any scene: include the StandardSurface kernels
        enqueue_bounces<4>(S->W, 0, kServeIters, false, &prof, sms, S->stream, true, true);
        e = cudaStreamEndCapture(S->stream, &g);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&S->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaFree(S->d_job_done);
        cudaFreeHost(S->h_done);
        cudaFreeHost(S->h_cnt);
        cudaFree(S->wave_mem);
        drop_streams();
        return cuda_status(ctx, e, "wave graph capture");
    }
    cudaStreamSynchronize(S->stream);
    Server *raw = S.release();
    ctx->children++;
    raw->worker = std::thread(worker_loop, raw);
    raw->builder = std::thread(builder_loop, raw);
    raw->reader = std::thread(reader_loop, raw);
    *out = reinterpret_cast<fl_server *>(raw);
    return FL_OK;
}

fl_status fl_server_destroy(fl_server *srv) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S) return FL_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_build.notify_all();
    if (S->worker.joinable()) S->worker.join();
    if (S->builder.joinable()) S->builder.join();
    S->cv_read.notify_all();
    if (S->reader.joinable()) S->reader.join();  // finishes the read-outs in flight
    if (S->tracing) {
        if (FILE *f = std::fopen(S->trace_path.c_str(), "a")) {
            std::fprintf(f, "# server policy %d\n", S->cfg.policy);
            for (const auto &l : S->trace) std::fprintf(f, "%s\n", l.c_str());
            std::fclose(f);
        }
    }
    cudaSetDevice(S->ctx->device);
    cudaStreamSynchronize(S->stream);
    for (const BuildTask &t : S->build_q)
        if (t.release) fl_scene_destroy(reinterpret_cast<fl_scene *>(t.release));
    for (auto &kv : S->jobs) {
        if (kv.second->d_film) cudaFreeAsync(kv.second->d_film, S->stream);
        if (kv.second->d_rgb) cudaFreeAsync(kv.second->d_rgb, S->stream);
        cudaFreeHost(kv.second->h_rgb);
        cudaFreeHost(kv.second->h_xyz);
    }
    cudaStreamSynchronize(S->stream);
    for (auto &kv : S->pinned_pool) cudaFreeHost(kv.second);
    for (cudaEvent_t e : S->free_events) cudaEventDestroy(e);
    for (auto &kv : S->scenes)
        if (kv.second.dev) fl_scene_destroy(reinterpret_cast<fl_scene *>(kv.second.dev));
    if (S->graph) cudaGraphExecDestroy(S->graph);
    cudaFree(S->d_job_done);
    cudaFreeHost(S->h_done);
    cudaFreeHost(S->h_cnt);
    cudaFree(S->wave_mem);
    cudaStreamSynchronize(S->rstream);
    cudaEventDestroy(S->ev_resolved);
    cudaStreamDestroy(S->rstream);
    cudaStreamDestroy(S->stream);
    S->ctx->children--;
    delete S;
    return FL_OK;
}

fl_status fl_server_add_scene(fl_server *srv, const fl_scene_desc *d, uint64_t *scene_id) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S || !d || !scene_id || !d->materials || d->n_materials == 0 || (d->n_tri && !d->verts) ||
        (d->n_lights && !d->lights))
        return FL_ERR_INVALID;
    if ((int)d->n_lights > S->cfg.max_lights) {
        set_error(S->ctx, "scene has more lights than the server was configured for");
        return FL_ERR_INVALID;
    }
    HostScene h;
    h.verts.assign(d->verts, d->verts + 9 * (size_t)d->n_tri);
    if (d->tri_material) h.tri_material.assign(d->tri_material, d->tri_material + d->n_tri);
    else h.tri_material.assign(d->n_tri, 0u);
    h.materials.assign(d->materials, d->materials + d->n_materials);
    if (d->n_lights) h.lights.assign(d->lights, d->lights + d->n_lights);
    if (d->standard_surfaces && d->n_standard_surfaces)
        h.standard.assign(d->standard_surfaces, d->standard_surfaces + d->n_standard_surfaces);
    if (d->uvs) h.uvs.assign(d->uvs, d->uvs + 6 * (size_t)d->n_tri);
    for (uint32_t i = 0; d->images && i < d->n_images; ++i) {
        const fl_image &im = d->images[i];
        if (im.width <= 0 || im.height <= 0 || !im.rgb || (uint64_t)im.width * im.height > (1ull << 28)) {
            set_error(S->ctx, "invalid image");
            return FL_ERR_INVALID;
        }
        h.pixels.emplace_back(im.rgb, im.rgb + 3 * (size_t)im.width * im.height);
    }
    for (size_t i = 0; i < h.pixels.size(); ++i)
        h.images.push_back(fl_image{d->images[i].width, d->images[i].height, h.pixels[i].data()});
    h.bytes = scene_bytes_estimate(d->n_tri, d->n_materials) + 4 * h.uvs.size() +
              (uint64_t)h.standard.size() * (sizeof(StandardDev) + sizeof(float) * kStdSpectra * 60);
    for (const auto &px : h.pixels) h.bytes += px.size();
    std::lock_guard<std::mutex> lock(S->mu);
    const uint64_t id = S->next_scene++;
    S->sched.add_scene(id, h.bytes);
    S->scenes[id] = std::move(h);
    *scene_id = id;
    return FL_OK;
}

fl_status fl_server_remove_scene(fl_server *srv, uint64_t scene_id) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S) return FL_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        auto it = S->scenes.find(scene_id);
        if (it == S->scenes.end() || it->second.removed) {
            set_error(S->ctx, "unknown scene id");
            return FL_ERR_INVALID;
        }
        it->second.removed = true;
        S->removals++;
        S->events++;
    }
    S->cv_work.notify_one();
    return FL_OK;
}

fl_status fl_server_submit(fl_server *srv, const fl_job_desc *job, uint64_t *job_id) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S || !job || !job_id) return FL_ERR_INVALID;
    const fl_camera &c = job->camera;
    const fl_render_params &p = job->params;
    if (!camera_ok(c) || p.spp <= 0 || !depths_ok(p) || deepest_depth(p) > S->cfg.max_depth ||
        p.spectral_mode != FL_SPECTRAL_HERO4) {
        set_error(S->ctx, "invalid job (hero-wavelength mode, depths within the server's max_depth)");
        return FL_ERR_INVALID;
    }
    auto hj = std::make_unique<HostJob>();
    hj->cam = c;
    hj->params = p;
    hj->scene = job->scene_id;
    const uint64_t film = (uint64_t)c.width * c.height * 3 * (sizeof(double) + sizeof(float));
    const uint64_t samples = (uint64_t)c.width * c.height * (uint64_t)p.spp;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        auto sc = S->scenes.find(job->scene_id);
        if (!S->sched.has_scene(job->scene_id) || sc == S->scenes.end() || sc->second.removed) {
            set_error(S->ctx, "unknown or removed scene id");
            return FL_ERR_INVALID;
        }
        const uint64_t id = S->next_job++;
        hj->submit_ms = S->now_ms();
        S->jobs[id] = std::move(hj);
        S->sched.submit(id, job->scene_id, film, samples);
        S->stats.jobs_submitted++;
        S->events++;
        *job_id = id;
    }
    S->cv_work.notify_one();
    return FL_OK;
}

static fl_status collect(Server *S, uint64_t job_id, float *film_rgb, double *film_xyz64, fl_job_stats *st) {
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) return FL_ERR_INVALID;
    HostJob &j = *it->second;
    if (j.status == FL_ERR_NOT_READY) return FL_ERR_NOT_READY;
    if (st) {
        st->submit_ms = j.submit_ms;
        st->start_ms = j.start_ms;
        st->done_ms = j.done_ms;
        st->samples = (uint64_t)j.cam.width * j.cam.height * (uint64_t)j.params.spp;
    }
    const fl_status rc = j.status;
    const size_t n_pix = (size_t)j.cam.width * j.cam.height;
    if (rc == FL_OK) {
        if (film_rgb) std::memcpy(film_rgb, j.h_rgb, n_pix * 3 * sizeof(float));
        if (film_xyz64) std::memcpy(film_xyz64, j.h_xyz, n_pix * 3 * sizeof(double));
    }
    S->release_pinned(j.h_rgb, n_pix * 3 * sizeof(float));
    S->release_pinned(j.h_xyz, n_pix * 3 * sizeof(double));
    S->jobs.erase(it);  // results are handed out once
    return rc;
}

fl_status fl_server_poll(fl_server *srv, uint64_t job_id, float *film_rgb, double *film_xyz64, fl_job_stats *st) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S) return FL_ERR_INVALID;
    std::lock_guard<std::mutex> lock(S->mu);
    return collect(S, job_id, film_rgb, film_xyz64, st);
}

fl_status fl_server_wait(fl_server *srv, uint64_t job_id, int32_t timeout_ms, float *film_rgb, double *film_xyz64,
                         fl_job_stats *st) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S) return FL_ERR_INVALID;
    std::unique_lock<std::mutex> lock(S->mu);
    auto ready = [&] {
        auto it = S->jobs.find(job_id);
        return it == S->jobs.end() || it->second->status != FL_ERR_NOT_READY;
    };
    if (timeout_ms < 0) S->cv_done.wait(lock, ready);
    else if (!S->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready)) return FL_ERR_TIMEOUT;
    return collect(S, job_id, film_rgb, film_xyz64, st);
}

fl_status fl_server_get_stats(fl_server *srv, fl_server_stats *st) {
    Server *S = reinterpret_cast<Server *>(srv);
    if (!S || !st) return FL_ERR_INVALID;
    std::lock_guard<std::mutex> lock(S->mu);
    *st = S->stats;
    st->resident_bytes = S->sched.used();
    st->running = (uint32_t)S->sched.running();
    st->pending = (uint32_t)S->sched.pending();
    return S->error.empty() ? FL_OK : FL_ERR_CUDA;
}

}  // extern "C"
