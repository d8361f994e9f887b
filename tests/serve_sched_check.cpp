// Drives the serving scheduler (filianore-core_b200/csrc/fl_serve_sched.h) through fixed
// scenarios and prints the decisions as text for tests/test_serve_sched.py.
#include <cstdio>

#include "../filianore-core_b200/csrc/fl_serve_sched.h"

using fl::ServeScheduler;

static void print_adm(const char *tag, const ServeScheduler::Admission &a) {
    std::printf("%s admitted", tag);
    for (auto j : a.admitted) std::printf(" %llu", (unsigned long long)j);
    std::printf(" | build");
    for (auto s : a.build) std::printf(" %llu", (unsigned long long)s);
    std::printf(" | evict");
    for (auto s : a.evict) std::printf(" %llu", (unsigned long long)s);
    std::printf(" | rejected");
    for (auto j : a.rejected) std::printf(" %llu", (unsigned long long)j);
    std::printf("\n");
}

static void print_plan(const char *tag, const std::vector<ServeScheduler::Seg> &p) {
    std::printf("%s", tag);
    for (auto &s : p) std::printf(" %llu:%u@%llu", (unsigned long long)s.job, s.count, (unsigned long long)s.sample_base);
    std::printf("\n");
}

int main() {
    // budget 1000: scenes 1 (400 B), 2 (500 B), 3 (300 B); films of 100 B
    ServeScheduler s(1000, 2);
    s.add_scene(1, 400);
    s.add_scene(2, 500);
    s.add_scene(3, 300);
    s.submit(10, 1, 100, 250);   // job 10 on scene 1, 250 samples
    s.submit(11, 2, 100, 100);   // job 11 on scene 2
    s.submit(12, 3, 100, 50);    // job 12 on scene 3: must wait (max_jobs 2 and memory)
    s.submit(13, 1, 2000, 10);   // job 13 can never fit
    print_adm("A1", s.admit());
    std::printf("used %llu\n", (unsigned long long)s.used());
    print_plan("P1", s.plan_wave(256));
    print_plan("P2", s.plan_wave(256));
    auto d = s.finish_wave();
    std::printf("done");
    for (auto j : d) std::printf(" %llu", (unsigned long long)j);
    std::printf("\n");
    print_adm("A2", s.admit());
    print_plan("P3", s.plan_wave(256));
    d = s.finish_wave();
    std::printf("done");
    for (auto j : d) std::printf(" %llu", (unsigned long long)j);
    std::printf("\n");
    print_adm("A3", s.admit());
    std::printf("used %llu idle %d\n", (unsigned long long)s.used(), (int)s.idle());

    // wave packing policies: jobs 20..23 (arrival order) with 300, 40, 200, 10 samples
    const char *names[] = {"shortest", "first_come", "fair", "aged", "ratio"};
    for (int pol = 0; pol < 5; ++pol) {
        ServeScheduler q(1 << 20, 8, pol);
        q.add_scene(1, 100);
        const uint64_t want[] = {300, 40, 200, 10};
        for (int j = 0; j < 4; ++j) q.submit(20 + j, 1, 10, want[j]);
        q.admit();
        print_plan(names[pol], q.plan_wave(256));
    }

    // response ratio over time: job 30 (2000 samples) waits while short jobs keep arriving;
    // its ratio grows with the waves it waits, until it is served ahead of a newcomer
    {
        ServeScheduler q(1 << 20, 8, ServeScheduler::kResponseRatio);
        q.add_scene(1, 100);
        q.submit(30, 1, 10, 2000);
        q.admit();
        uint64_t next = 31;
        for (int w = 0; w < 10; ++w) {
            q.submit(next++, 1, 10, 200);  // one short job per wave
            q.admit();
            auto p = q.plan_wave(256);
            std::printf("R%d", w);
            for (auto &sg : p) std::printf(" %llu:%u", (unsigned long long)sg.job, sg.count);
            std::printf("\n");
            q.finish_wave();
        }
    }
    // a resident, idle scene whose bytes plus the job's film exceed the budget: the job can
    // never run (it holds both), so it is rejected instead of waiting forever at the head
    {
        ServeScheduler q(100, 4);
        q.add_scene(1, 60);
        q.submit(40, 1, 30, 10);  // fits: 60 + 30
        print_adm("B1", q.admit());
        q.plan_wave(64);
        q.finish_wave();
        q.submit(41, 1, 50, 10);  // 60 + 50 > 100 with the scene already resident
        q.submit(42, 1, 20, 10);  // behind it, fits
        print_adm("B2", q.admit());
        std::printf("pending %d running %d\n", (int)q.pending(), (int)q.running());
    }
    // earliest deadline first: job 50 (2000 samples, deadline 0 + 1 + 2 x 2000/256 = 16.6)
    // waits behind short jobs arriving each wave (deadline w + 1 + 2 x 200/256 = w + 2.6)
    // until their deadlines pass its own, then takes whole waves
    {
        ServeScheduler q(1 << 20, 8, ServeScheduler::kDeadline);
        q.add_scene(1, 100);
        q.submit(50, 1, 10, 2000);
        q.admit();
        uint64_t next = 51;
        for (int w = 0; w < 18; ++w) {
            q.submit(next++, 1, 10, 200);
            q.admit();
            auto p = q.plan_wave(256);
            std::printf("D%d", w);
            for (auto &sg : p) std::printf(" %llu:%u", (unsigned long long)sg.job, sg.count);
            std::printf("\n");
            q.finish_wave();
        }
    }
    // arrival order with a small-job lane: job 70 (2000 samples) and job 71 (200) arrive with
    // job 72 (10); a 20-sample job arrives every later wave. The small jobs take the lane (an
    // eighth of 256 = 32), the rest of each wave goes to 70 until it is done, then to 71.
    {
        ServeScheduler q(1 << 20, 16, ServeScheduler::kFirstComeLane);
        q.add_scene(1, 100);
        q.submit(70, 1, 10, 2000);
        q.submit(71, 1, 10, 200);
        q.submit(72, 1, 10, 10);
        uint64_t next = 73;
        for (int w = 0; w < 9; ++w) {
            if (w > 0) q.submit(next++, 1, 10, 20);
            q.admit();
            auto p = q.plan_wave(256);
            std::printf("L%d", w);
            for (auto &sg : p) std::printf(" %llu:%u", (unsigned long long)sg.job, sg.count);
            std::printf("\n");
            q.finish_wave();
        }
    }
    // asynchronous builds: a job whose scene is still being built gets no samples; jobs with
    // ready scenes take the wave meanwhile
    {
        ServeScheduler q(1 << 20, 8, ServeScheduler::kFirstCome);
        q.set_async_builds(true);
        q.add_scene(1, 100);
        q.add_scene(2, 100);
        q.submit(80, 1, 10, 100);
        auto a = q.admit();
        auto p = q.plan_wave(256);
        std::printf("G1 build %d planned %d ready %d\n", (int)a.build.size(), (int)p.size(), (int)q.scene_ready(1));
        q.finish_wave();
        q.scene_built(1);
        q.submit(81, 2, 10, 100);
        a = q.admit();
        print_plan("G2", q.plan_wave(256));
        q.finish_wave();
        q.scene_built(2);
        q.submit(82, 2, 10, 50);
        q.admit();
        print_plan("G3", q.plan_wave(256));
    }
    // completing single jobs (the streaming server): only a running job with every sample
    // dispatched completes; its film and its hold on the scene are released
    {
        ServeScheduler q(1000, 4, ServeScheduler::kFirstCome);
        q.add_scene(1, 300);
        q.submit(90, 1, 50, 100);
        q.submit(91, 1, 50, 300);
        q.admit();
        q.plan_wave(256);  // 90: 100, 91: 156 of 300
        const int a90 = q.dispatched_all(90), a91 = q.dispatched_all(91);
        const int c91 = q.complete(91), c90 = q.complete(90);
        std::printf("H1 %d %d %d %d used %llu\n", a90, a91, c91, c90, (unsigned long long)q.used());
        q.plan_wave(256);  // 91: the other 144
        const int b91 = q.dispatched_all(91), d91 = q.complete(91);
        std::printf("H2 %d %d running %d used %llu unused %d\n", b91, d91, (int)q.running(),
                    (unsigned long long)q.used(), (int)q.scene_unused(1));
    }
    // forgetting a scene: only once no pending or running job uses it; its bytes are released
    {
        ServeScheduler q(1000, 4);
        q.add_scene(1, 300);
        q.submit(60, 1, 10, 10);
        q.admit();
        std::printf("F unused %d used %llu\n", (int)q.scene_unused(1), (unsigned long long)q.used());
        q.plan_wave(64);
        q.finish_wave();
        std::printf("F unused %d\n", (int)q.scene_unused(1));
        const int was_resident = (int)q.forget_scene(1);
        std::printf("F resident %d used %llu known %d\n", was_resident, (unsigned long long)q.used(),
                    (int)q.has_scene(1));
    }
    return 0;
}
