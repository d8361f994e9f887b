"""The render server (fl_server_*): jobs on different scenes, resolutions and spp rendered
together in shared waves give the same images as rendering each alone with fl_render
(identical per-sample streams; only the FP64 film summation order differs), including
after LRU eviction and rebuild of a scene."""
import numpy as np
import pytest

import filianore_b200 as fb
from filianore_b200 import scenes

pytestmark = pytest.mark.gpu


def alone(ctx, sc, cam, p):
    s = ctx.scene(sc)
    xyz = np.zeros((cam.height, cam.width, 3), np.float64)
    rgb, _ = s.render(p, camera=cam, film_xyz64=xyz)
    s.close()
    return rgb, xyz


def test_mixed_jobs_equal_alone():
    ctx = fb.Context(0)
    srv = fb.Server(ctx, budget_bytes=2 << 30, max_depth=8, max_jobs=8, max_lights=4, wave_paths=1 << 16)
    scs = [scenes.cornell(64, 48, "materials"), scenes.cornell(96, 96),
           scenes.procedural_spheres(n_spheres=6, slices=32, stacks=17, width=80, height=60, extent=3.0,
                                     sphere_light=(0.0, 3.0, 0.0, 0.5, 40.0))]
    ids = [srv.add_scene(sc) for sc in scs]
    jobs = []
    for k, (sid, sc, spp) in enumerate(zip(ids, scs, (16, 4, 8))):
        cam = sc.camera_struct()
        p = scenes.render_params(spp, 8, fb.FL_SPECTRAL_HERO4)
        jobs.append((srv.submit(sid, cam, p), sc, cam, p))
    # a second job on the first scene with another camera size joins the mix
    cam2 = scs[0].camera_struct(40, 40)
    p2 = scenes.render_params(6, 8, fb.FL_SPECTRAL_HERO4)
    jobs.append((srv.submit(ids[0], cam2, p2), scs[0], cam2, p2))
    for jid, sc, cam, p in jobs:
        rgb, xyz, st = srv.wait(jid, timeout_ms=60000, want_xyz=True)
        want_rgb, want_xyz = alone(ctx, sc, cam, p)
        np.testing.assert_allclose(xyz, want_xyz, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(rgb, want_rgb, rtol=1e-5, atol=1e-6)
        assert st["done_ms"] >= st["start_ms"] >= st["submit_ms"]
    stats = srv.stats()
    assert stats["jobs_done"] == 4 and stats["builds"] == 3
    srv.close()
    ctx.close()


def test_eviction_and_rebuild_keep_results():
    """a budget that holds one scene at a time forces eviction and rebuild"""
    ctx = fb.Context(0)
    a = scenes.procedural_spheres(n_spheres=4, slices=64, stacks=33, width=48, height=32, extent=3.0)
    b = scenes.cornell(48, 32)
    # the server's footprint estimate: 132 B per triangle + 300 B per material + 1 MiB per
    # scene, 36 B per film pixel; the budget holds scene a and one film but not b as well
    est = lambda sc: sc.n_tri * 132 + len(sc.materials) * 300 + (1 << 20)  # noqa: E731
    budget = est(a) + 48 * 32 * 36 + est(b) // 2
    srv = fb.Server(ctx, budget_bytes=budget, max_depth=8, max_jobs=4, max_lights=4, wave_paths=1 << 14)
    ia, ib = srv.add_scene(a), srv.add_scene(b)
    order = [(ia, a), (ib, b), (ia, a)]
    ids = []
    for sid, sc in order:
        p = scenes.render_params(4, 8, fb.FL_SPECTRAL_HERO4)
        ids.append((srv.submit(sid, sc.camera_struct(), p), sc, p))
    for jid, sc, p in ids:
        _, xyz, _ = srv.wait(jid, timeout_ms=60000, want_xyz=True)
        _, want = alone(ctx, sc, sc.camera_struct(), p)
        np.testing.assert_allclose(xyz, want, rtol=1e-9, atol=1e-12)
    st = srv.stats()
    assert st["evictions"] >= 2 and st["builds"] >= 3
    srv.close()
    ctx.close()


def test_job_too_large_is_rejected():
    ctx = fb.Context(0)
    sc = scenes.cornell(32, 32)
    srv = fb.Server(ctx, budget_bytes=1 << 20, max_depth=8, max_jobs=2, max_lights=4, wave_paths=1 << 12)
    sid = srv.add_scene(sc)
    jid = srv.submit(sid, sc.camera_struct(4096, 4096), scenes.render_params(1, 8, fb.FL_SPECTRAL_HERO4))
    with pytest.raises(fb.FlError) as e:
        srv.wait(jid, timeout_ms=30000)
    assert e.value.status == fb.FL_ERR_CAPACITY
    srv.close()
    ctx.close()


def test_served_standard_surface_and_textures_equal_plain_render():
    """Scenes with StandardSurface materials (thin walls, measured copper under a thin film,
    with the measured metal curves), image textures and bump maps, served in one mix: the
    server keeps its own copies of the StandardSurface records, texture coordinates and
    images, and each job's image equals fl_render's."""
    ctx = fb.Context(0, tables=fb.reference_tables(measured_metals=True))
    srv = fb.Server(ctx, budget_bytes=2 << 30, max_depth=8, max_jobs=8, max_lights=4, wave_paths=1 << 16)
    scs = [scenes.cornell_textured(48, 48, bump=True), scenes.cornell(40, 40, "standard3"),
           scenes.cornell(40, 40, "standard")]
    ids = [srv.add_scene(sc) for sc in scs]   # the scene objects' buffers may go after this
    jobs = []
    for sid, sc, spp in zip(ids, scs, (8, 6, 4)):
        cam = sc.camera_struct()
        p = scenes.render_params(spp, 8, fb.FL_SPECTRAL_HERO4)
        jobs.append((srv.submit(sid, cam, p), sc, cam, p))
    for jid, sc, cam, p in jobs:
        rgb, xyz, _ = srv.wait(jid, timeout_ms=60000, want_xyz=True)
        want_rgb, want_xyz = alone(ctx, sc, cam, p)
        assert want_xyz.mean() > 0
        np.testing.assert_allclose(xyz, want_xyz, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(rgb, want_rgb, rtol=1e-5, atol=1e-6)
    srv.close()
    ctx.close()


def test_unequal_lobe_depths_and_many_refills_equal_alone():
    """Jobs with unequal lobe depths (paths may outlive the deepest depth) on a server of 2,048
    path slots, so that every job's paths stream through the slots over many iterations and
    share them with the other jobs: the images equal fl_render's for each job alone."""
    ctx = fb.Context(0)
    srv = fb.Server(ctx, budget_bytes=2 << 30, max_depth=8, max_jobs=8, max_lights=4, wave_paths=2048)
    sc_a = scenes.cornell(48, 40, "standard2")
    sc_b = scenes.cornell(32, 32, "materials")
    ia, ib = srv.add_scene(sc_a), srv.add_scene(sc_b)
    jobs = []
    for sid, sc, spp, depths in ((ia, sc_a, 6, (5, 3, 6)), (ib, sc_b, 4, (3, 6, 5)), (ia, sc_a, 2, (2, 7, 4))):
        cam = sc.camera_struct()
        p = scenes.render_params(spp, 8, fb.FL_SPECTRAL_HERO4, depths=depths)
        jobs.append((srv.submit(sid, cam, p), sc, cam, p))
    for jid, sc, cam, p in jobs:
        _, xyz, _ = srv.wait(jid, timeout_ms=60000, want_xyz=True)
        _, want = alone(ctx, sc, cam, p)
        np.testing.assert_allclose(xyz, want, rtol=1e-9, atol=1e-12)
    assert srv.stats()["jobs_done"] == 3
    srv.close()
    ctx.close()
