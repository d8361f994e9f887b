// Serving scheduler (host only, no CUDA): admission of render jobs by memory footprint,
// scene residency with least-recently-used eviction, and the planning of shared waves.
//
// Policy:
//  - Jobs are admitted first come, first served while (a) fewer than max_jobs run and
//    (b) the job's film plus, when its scene is not resident, the scene fit the memory
//    budget. To make room, resident scenes that no running or admitted job uses are
//    evicted, least recently used first. The queue head blocks later jobs (no reordering),
//    so admission order is arrival order. A job that could never fit is rejected.
//  - Each wave is packed shortest-remaining-first (the default policy): running jobs are taken in order of
//    the samples they still have to render and each takes as many of the wave's path
//    slots as it can use. Small jobs finish within a wave or two; large jobs fill the
//    rest of every wave, so the GPU stays full. (A simulation of this workload's Poisson
//    load favoured this over first-come-first-served packing, equal sharing and a
//    reserved share for the oldest job, at both the median and the 99th percentile.)
//    The other policies are first come, first served packing, equal sharing
//    (water-filling), shortest-remaining-first with a quarter of every wave reserved for
//    the oldest running job, highest response ratio next ((waves waited + waves needed) /
//    waves needed), earliest deadline first (deadline = submission + 2 x the waves the job
//    needs alone + 1), and arrival order with an eighth of each wave reserved for small
//    jobs, shortest first. Each job gets one contiguous sample range per wave, so its
//    per-sample random streams do not depend on how it was batched.
//  - A job is complete when all its samples were dispatched and the wave that carried its
//    last samples has finished.
#pragma once

#include <algorithm>
#include <cstdint>
#include <deque>
#include <map>
#include <vector>

namespace fl {

class ServeScheduler {
public:
    struct Seg {
        uint64_t job;
        uint32_t count;
        uint64_t sample_base;
    };
    struct Admission {
        std::vector<uint64_t> admitted;  // jobs that start running
        std::vector<uint64_t> build;     // scenes to make resident (before the admitted jobs run)
        std::vector<uint64_t> evict;     // scenes to release
        std::vector<uint64_t> rejected;  // jobs that can never fit the budget
    };

    enum Policy {
        kShortestFirst = 0,
        kFirstCome = 1,
        kFairShare = 2,
        kShortestFirstAged = 3,
        kResponseRatio = 4,
        kDeadline = 5,
        kFirstComeLane = 6
    };
    // kFirstComeLane: an eighth of every wave is a lane for small jobs (those that need no
    // more than the lane), shortest first; the rest of the wave goes to the running jobs in
    // arrival order. A large job then runs at seven eighths of the GPU at least, in arrival
    // order, while small jobs do not queue behind it.
    static constexpr uint32_t kLaneDivisor = 8;
    // kDeadline: a job's deadline is its submission (in planned waves) plus kDeadlineSlack times
    // the waves it needs alone, plus one; waves go to the earliest deadlines first. Small jobs
    // get near deadlines and pass large ones, but a large job's deadline does not move, so
    // once it is the earliest it is served ahead of every later arrival.
    static constexpr double kDeadlineSlack = 2.0;

    ServeScheduler(uint64_t budget_bytes, int max_jobs, int policy = kShortestFirst)
        : budget_(budget_bytes), max_jobs_(max_jobs), policy_(policy) {}

    void add_scene(uint64_t id, uint64_t bytes) { scenes_[id] = SceneState{bytes, false, 0, 0, false}; }
    // With asynchronous builds a scene that admission makes resident is not ready until
    // scene_built(id): its jobs are admitted (their memory is reserved) but get no samples
    // until then, while jobs whose scenes are ready keep the waves full. Without them a
    // resident scene is ready at once (the caller builds it before the next wave).
    void set_async_builds(bool on) { async_builds_ = on; }
    // kFirstComeLane's lane (share of a wave) and the largest job it takes (in waves);
    // 0 keeps the defaults (an eighth of the wave, for jobs that fit in it)
    void set_lane(double share, double small_waves) {
        lane_share_ = share;
        lane_small_waves_ = small_waves;
    }
    void scene_built(uint64_t id) {
        auto it = scenes_.find(id);
        if (it != scenes_.end() && it->second.resident) it->second.built = true;
    }
    bool scene_ready(uint64_t id) const {
        auto it = scenes_.find(id);
        return it != scenes_.end() && it->second.resident && it->second.built;
    }
    bool has_scene(uint64_t id) const { return scenes_.count(id) != 0; }
    bool scene_resident(uint64_t id) const {
        auto it = scenes_.find(id);
        return it != scenes_.end() && it->second.resident;
    }

    void submit(uint64_t job, uint64_t scene, uint64_t film_bytes, uint64_t total_samples) {
        jobs_[job] = JobState{scene, film_bytes, total_samples, 0, false, false, waves_};
        pending_.push_back(job);
    }

    Admission admit() {
        Admission a;
        while (!pending_.empty() && (int)running_.size() < max_jobs_) {
            const uint64_t j = pending_.front();
            JobState &js = jobs_[j];
            SceneState &sc = scenes_[js.scene];
            const uint64_t need = js.film_bytes + (sc.resident ? 0 : sc.bytes);
            // The job holds its scene and its film for as long as it runs, so scene + film
            // beyond the budget can never fit, whether or not the scene is resident now.
            if (js.film_bytes + sc.bytes > budget_) {
                a.rejected.push_back(j);
                pending_.pop_front();
                jobs_.erase(j);
                continue;
            }
            if (used_ + need > budget_) {
                // evict idle resident scenes, least recently used first
                std::vector<std::pair<uint64_t, uint64_t>> idle;  // (last_use, scene)
                for (auto &kv : scenes_)
                    if (kv.second.resident && kv.second.users == 0 && kv.first != js.scene)
                        idle.push_back({kv.second.last_use, kv.first});
                std::sort(idle.begin(), idle.end());
                uint64_t freeable = 0;
                for (auto &p : idle) freeable += scenes_[p.second].bytes;
                if (used_ + need > budget_ + freeable) break;  // wait for running jobs to finish
                for (auto &p : idle) {
                    if (used_ + need <= budget_) break;
                    SceneState &ev = scenes_[p.second];
                    ev.resident = false;
                    ev.built = false;
                    used_ -= ev.bytes;
                    a.evict.push_back(p.second);
                }
            }
            if (!sc.resident) {
                sc.resident = true;
                sc.built = !async_builds_;
                used_ += sc.bytes;
                a.build.push_back(js.scene);
            }
            used_ += js.film_bytes;
            sc.users += 1;
            sc.last_use = ++clock_;
            js.running = true;
            running_.push_back(j);
            a.admitted.push_back(j);
            pending_.pop_front();
        }
        return a;
    }

    // Splits `cap` slots over running jobs that still have samples to dispatch and whose
    // scenes are ready.
    std::vector<Seg> plan_wave(uint32_t cap) {
        std::vector<std::pair<uint64_t, uint64_t>> want;  // (remaining, job)
        for (uint64_t j : running_) {
            const JobState &js = jobs_[j];
            if (js.dispatched < js.total && scene_ready(js.scene)) want.push_back({js.total - js.dispatched, j});
        }
        std::vector<Seg> segs;
        uint64_t left = cap;
        if (policy_ == kFairShare) {
            // water-filling: jobs needing less than an equal share get all they need
            std::sort(want.begin(), want.end());
            size_t n = want.size();
            for (size_t i = 0; i < want.size() && left > 0; ++i, --n) {
                const uint64_t g = std::min<uint64_t>(want[i].first, std::max<uint64_t>(left / n, 1));
                JobState &js = jobs_[want[i].second];
                segs.push_back(Seg{want[i].second, (uint32_t)g, js.dispatched});
                js.dispatched += g;
                left -= g;
            }
        } else {
            if (policy_ == kShortestFirstAged && !want.empty()) {
                // the oldest running job (running_ is in arrival order) is guaranteed a
                // quarter of the wave, which bounds how long shorter arrivals can starve it
                const uint64_t g = std::min<uint64_t>(want[0].first, cap / 4);
                JobState &js = jobs_[want[0].second];
                segs.push_back(Seg{want[0].second, (uint32_t)g, js.dispatched});
                js.dispatched += g;
                left -= g;
                want[0].first -= g;
                if (want[0].first == 0) want.erase(want.begin());
            }
            if (policy_ == kFirstComeLane) {
                std::vector<std::pair<uint64_t, uint64_t>> small;
                const uint64_t lane = lane_share_ > 0.0 ? (uint64_t)(lane_share_ * cap) : cap / kLaneDivisor;
                const uint64_t small_max = lane_small_waves_ > 0.0 ? (uint64_t)(lane_small_waves_ * cap) : lane;
                for (auto &w : want)
                    if (w.first <= small_max) small.push_back(w);
                std::stable_sort(small.begin(), small.end(),
                                 [](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
                                     return a.first < b.first;
                                 });
                uint64_t lane_left = lane;
                for (auto &w : small) {
                    if (lane_left == 0) break;
                    const uint64_t g = std::min<uint64_t>(w.first, lane_left);
                    JobState &js = jobs_[w.second];
                    segs.push_back(Seg{w.second, (uint32_t)g, js.dispatched});
                    js.dispatched += g;
                    lane_left -= g;
                    left -= g;
                }
                for (auto &w : want) w.first = jobs_[w.second].total - jobs_[w.second].dispatched;
                want.erase(std::remove_if(want.begin(), want.end(),
                                          [](const std::pair<uint64_t, uint64_t> &w) { return w.first == 0; }),
                           want.end());
                // the rest in arrival order (want follows running_, which is in arrival order)
            } else if (policy_ == kDeadline) {
                auto deadline = [&](const std::pair<uint64_t, uint64_t> &w) {
                    const JobState &js = jobs_[w.second];
                    return (double)js.submit_wave + 1.0 + kDeadlineSlack * (double)js.total / (double)cap;
                };
                std::stable_sort(want.begin(), want.end(),
                                 [&](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
                                     return deadline(a) < deadline(b);
                                 });
            } else if (policy_ == kResponseRatio) {
                // highest response ratio next: (waves waited, this one included, + waves still
                // needed) / waves still needed, so short jobs go first and a long job's
                // priority grows while it waits
                auto ratio = [&](const std::pair<uint64_t, uint64_t> &w) {
                    const double need = std::max(1.0, (double)w.first / (double)cap);
                    return ((double)(waves_ - jobs_[w.second].submit_wave + 1) + need) / need;
                };
                std::stable_sort(want.begin(), want.end(),
                                 [&](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
                                     return ratio(a) > ratio(b);
                                 });
            } else if (policy_ != kFirstCome && policy_ != kFirstComeLane) {
                // shortest remaining first (first come first served keeps running_'s arrival order)
                std::stable_sort(want.begin(), want.end(),
                                 [](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
                                     return a.first < b.first;
                                 });
            }
            for (size_t i = 0; i < want.size() && left > 0; ++i) {
                const uint64_t g = std::min<uint64_t>(want[i].first, left);
                JobState &js = jobs_[want[i].second];
                auto same = std::find_if(segs.begin(), segs.end(), [&](const Seg &q) { return q.job == want[i].second; });
                if (same != segs.end())
                    same->count += (uint32_t)g;  // the oldest job's reserved range continues
                else
                    segs.push_back(Seg{want[i].second, (uint32_t)g, js.dispatched});
                js.dispatched += g;
                left -= g;
            }
        }
        ++waves_;
        // keep admission (arrival) order inside the wave
        std::sort(segs.begin(), segs.end(), [&](const Seg &a, const Seg &b) { return order(a.job) < order(b.job); });
        return segs;
    }

    // Called when the last planned wave has finished: returns the jobs now complete and
    // releases their film and their hold on the scene.
    std::vector<uint64_t> finish_wave() {
        std::vector<uint64_t> done;
        for (auto it = running_.begin(); it != running_.end();) {
            JobState &js = jobs_[*it];
            if (js.dispatched >= js.total) {
                done.push_back(*it);
                used_ -= js.film_bytes;
                SceneState &sc = scenes_[js.scene];
                sc.users -= 1;
                sc.last_use = ++clock_;
                jobs_.erase(*it);
                it = running_.erase(it);
            } else {
                ++it;
            }
        }
        return done;
    }

    // Completes one running job whose samples were all dispatched and have all finished
    // (the streaming server learns that from the device): releases its film and its hold
    // on the scene. Returns false for a job that is not running or has samples left.
    bool complete(uint64_t job) {
        auto it = std::find(running_.begin(), running_.end(), job);
        if (it == running_.end()) return false;
        JobState &js = jobs_[job];
        if (js.dispatched < js.total) return false;
        used_ -= js.film_bytes;
        SceneState &sc = scenes_[js.scene];
        sc.users -= 1;
        sc.last_use = ++clock_;
        jobs_.erase(job);
        running_.erase(it);
        return true;
    }
    // whether every sample of a running job has been dispatched
    bool dispatched_all(uint64_t job) const {
        auto it = jobs_.find(job);
        return it != jobs_.end() && it->second.dispatched >= it->second.total;
    }

    // A scene no pending or running job uses (it may still be resident): can be forgotten.
    bool scene_unused(uint64_t id) const {
        auto it = scenes_.find(id);
        if (it == scenes_.end() || it->second.users != 0) return false;
        for (uint64_t j : pending_) {
            auto jt = jobs_.find(j);
            if (jt != jobs_.end() && jt->second.scene == id) return false;
        }
        return true;
    }
    // Forgets an unused scene; returns whether it was resident (its memory is released).
    bool forget_scene(uint64_t id) {
        auto it = scenes_.find(id);
        if (it == scenes_.end()) return false;
        const bool resident = it->second.resident;
        if (resident) used_ -= it->second.bytes;
        scenes_.erase(it);
        return resident;
    }

    uint64_t used() const { return used_; }
    size_t running() const { return running_.size(); }
    size_t pending() const { return pending_.size(); }
    bool idle() const { return running_.empty() && pending_.empty(); }
    const std::vector<uint64_t> &running_jobs() const { return running_; }

private:
    struct SceneState {
        uint64_t bytes;
        bool resident;
        uint64_t last_use;
        int users;
        bool built;  // resident and ready for rendering
    };
    struct JobState {
        uint64_t scene, film_bytes, total, dispatched;
        bool running, done;
        uint64_t submit_wave;  // waves planned before the job was submitted
    };
    size_t order(uint64_t j) const {
        return (size_t)(std::find(running_.begin(), running_.end(), j) - running_.begin());
    }

    uint64_t budget_;
    int max_jobs_;
    int policy_;
    uint64_t used_ = 0;
    uint64_t clock_ = 0;
    uint64_t waves_ = 0;
    bool async_builds_ = false;
    double lane_share_ = 0.0, lane_small_waves_ = 0.0;
    std::map<uint64_t, SceneState> scenes_;
    std::map<uint64_t, JobState> jobs_;
    std::deque<uint64_t> pending_;
    std::vector<uint64_t> running_;
};

}  // namespace fl
