"""Host-side policy of the render server (no GPU): admission in arrival order by memory
footprint, LRU eviction of idle scenes, rejection of jobs that can never fit, and the
wave packing policies."""
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def run_driver():
    exe = os.path.join(tempfile.mkdtemp(), "serve_sched_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", exe, os.path.join(HERE, "serve_sched_check.cpp")], check=True)
    return subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines()


def test_scheduler_decisions():
    out = run_driver()
    # budget 1000: scene 1 (400) + film (100) fits; job 11 would need scene 2 (500) + film
    # on top of that (1100 > 1000), so it waits and blocks the queue behind it
    assert out[0] == "A1 admitted 10 | build 1 | evict | rejected"
    assert out[1] == "used 500"
    # a single running job gets the whole wave until all its samples are dispatched
    assert out[2] == "P1 10:250@0"
    assert out[3] == "P2"
    assert out[4] == "done 10"
    # scene 1 is now idle and is evicted (least recently used) to make room for scenes 2
    # and 3; max_jobs = 2 stops admission before job 13
    assert out[5] == "A2 admitted 11 12 | build 2 3 | evict 1 | rejected"
    # water-filling: job 12 (50 samples) gets all of its samples, job 11 the rest
    assert out[6] == "P3 11:100@0 12:50@0"
    assert out[7] == "done 11 12"
    # job 13's film alone exceeds the budget: rejected when it reaches the queue head
    assert out[8] == "A3 admitted | build | evict | rejected 13"
    assert out[9] == "used 800 idle 1"


def test_wave_packing_policies():
    out = run_driver()[10:]
    # shortest remaining first: the three short jobs complete, the long one fills the rest
    assert out[0] == "shortest 20:6@0 21:40@0 22:200@0 23:10@0"
    # arrival order: the oldest job takes the whole wave
    assert out[1] == "first_come 20:256@0"
    # water-filling: 10 and 40 fit an equal share, the other two split the remaining 206
    assert out[2] == "fair 20:103@0 21:40@0 22:103@0 23:10@0"
    # the oldest job keeps a quarter of the wave (64), the rest goes shortest first
    assert out[3] == "aged 20:64@0 21:40@0 22:142@0 23:10@0"
    # response ratio on the first wave (nobody has waited yet): shortest first
    assert out[4] == "ratio 20:6@0 21:40@0 22:200@0 23:10@0"


def test_response_ratio_bounds_waiting():
    """A long job (2000 samples) while one short job (200) arrives every wave of 256: each
    short job is served in the wave it arrives, the long one gets the rest, and once the long
    job has waited long enough it takes a whole wave ahead of the newcomer."""
    out = run_driver()[15:]
    assert out[:6] == [f"R{w} 30:56 {31 + w}:200" for w in range(6)]
    assert out[6] == "R6 30:256"
    assert out[7] == "R7 30:56 37:200"


def test_resident_scene_plus_film_over_budget_is_rejected():
    """Budget 100, scene 60: after a job with a 30-byte film finished, the scene stays
    resident and idle. A job with a 50-byte film can never run (it needs both, 110 bytes), so
    it is rejected rather than left blocking the queue; the job behind it is admitted."""
    out = run_driver()[25:]
    assert out[0] == "B1 admitted 40 | build 1 | evict | rejected"
    assert out[1] == "B2 admitted 42 | build | evict | rejected 41"
    assert out[2] == "pending 0 running 1"


def test_deadline_policy_serves_a_long_job_once_its_deadline_is_earliest():
    """Earliest deadline first: a 2000-sample job (deadline 1 + 2 x 2000 / 256 = 16.6 waves)
    shares each wave with a short job arriving every wave (deadline w + 1 + 2 x 200 / 256)
    while the short ones' deadlines are earlier, then takes whole waves: its wait is bounded
    by its own size, not by the arrivals behind it."""
    out = run_driver()[28:]
    assert out[:15] == [f"D{w} 50:56 {51 + w}:200" for w in range(15)]
    assert out[15:18] == [f"D{w} 50:256" for w in (15, 16, 17)]


def test_removed_scene_is_forgotten_only_when_unused():
    out = run_driver()[60:]
    assert out[0] == "F unused 0 used 310"      # a running job holds it
    assert out[1] == "F unused 1"               # the job is done
    assert out[2] == "F resident 1 used 0 known 0"


def test_first_come_lane_keeps_small_jobs_out_of_the_queue():
    """Arrival order with an eighth of each wave (32 of 256) reserved for jobs that fit in it:
    the small jobs finish in the wave they arrive, the 2000-sample job takes the other 7/8 in
    arrival order, and the 200-sample job (too large for the lane) waits behind it."""
    out = run_driver()[46:55]
    # (segments are listed in arrival order)
    assert out[0] == "L0 70:246 72:10"
    assert out[1:8] == [f"L{w} 70:236 {72 + w}:20" for w in range(1, 8)]
    assert out[8] == "L8 70:102 71:134 80:20"


def test_async_builds_hold_jobs_until_their_scene_is_built():
    """With asynchronous builds a job takes part in waves only once its scene is built: the
    first wave is empty while scene 1 builds; then job 80 renders alone while scene 2 builds;
    then 81 and 82 (scene 2, already resident and built: no new build) join."""
    out = run_driver()[55:58]
    assert out[0] == "G1 build 1 planned 0 ready 0"
    assert out[1] == "G2 80:100@0"
    assert out[2] == "G3 81:100@0 82:50@0"


def test_complete_releases_a_job_once_all_its_samples_are_dispatched():
    """The streaming server completes jobs one at a time when the device has finished their
    paths: a job with samples still to dispatch is not completed; a completed one releases
    its film (used 400 = scene 300 + the other film) and, with the last job, the scene's
    hold (the scene stays resident and becomes unused)."""
    out = run_driver()[58:60]
    assert out[0] == "H1 1 0 0 1 used 350"
    assert out[1] == "H2 1 1 running 0 used 300 unused 1"
