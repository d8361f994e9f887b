"""Edge cases of the B200 path through the C ABI, against the CPU oracle: empty batches,
degenerate rays (zero, NaN and infinite components, tmin >= tmax), hits exactly at tmin and
tmax, degenerate and coincident triangles (ties resolve to the lowest id), axis-aligned
rays, and renders of tiny images, depth 0 and scenes without lights."""
import numpy as np
import pytest

import oracle
import filianore_b200 as fb
from filianore_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fb.Context(0)
    yield c
    c.close()


def soup_scene(tris):
    return scenes.Scene(np.ascontiguousarray(tris, np.float32), np.zeros(tris.shape[0], np.uint32),
                        [{"type": fb.FL_MAT_LAMBERT, "rgb": (0.5, 0.5, 0.5)}], [], None)


def assert_same(gpu, cpu):
    assert np.array_equal(gpu["id"], cpu["id"]), np.flatnonzero(gpu["id"] != cpu["id"])[:10]
    hit = cpu["id"] >= 0
    for k in ("t", "u", "v"):
        assert np.array_equal(gpu[k][hit], cpu[k][hit]), k


def test_zero_rays(ctx):
    s = ctx.scene(soup_scene(scenes.triangle_soup(64, seed=1)))
    empty = np.zeros((0, 4), np.float32)
    assert s.trace_closest(empty, empty).shape == (0,)
    assert s.trace_occluded(empty, empty).shape == (0,)
    s.close()


def test_tmin_tmax_are_exclusive(ctx):
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    org = np.array([[0.2, 0.2, -1, 0], [0.2, 0.2, -1, 1.0], [0.2, 0.2, -1, 0]], np.float32)
    dirs = np.array([[0, 0, 1, 1.0], [0, 0, 1, np.inf], [0, 0, 1, 1.0000001]], np.float32)
    s = ctx.scene(soup_scene(tri))
    h = s.trace_closest(org, dirs)
    assert list(h["id"]) == [-1, -1, 0]
    assert_same(h, oracle.CpuBVH(tri).trace(org, dirs))
    s.close()


def test_degenerate_rays(ctx):
    tris = scenes.triangle_soup(2000, seed=3, sigma=0.05)
    nan, inf = np.nan, np.inf
    org = np.array([[0.5, 0.5, -1, 0], [nan, 0.5, 0.5, 0], [0.5, 0.5, 0.5, 0], [inf, 0.5, 0.5, 0],
                    [0.5, 0.5, -1, 2.0], [0.5, 0.5, -1, 0], [0.5, 0.5, -1, nan]], np.float32)
    dirs = np.array([[0, 0, 0, inf], [0, 0, 1, inf], [nan, 0, 1, inf], [-1, 0, 0, inf],
                     [0, 0, 1, 1.0], [0, 0, 1, -1.0], [0, 0, 1, inf]], np.float32)
    s = ctx.scene(soup_scene(tris))
    h = s.trace_closest(org, dirs)
    assert_same(h, oracle.CpuBVH(tris).trace(org, dirs))
    assert np.all(h["id"][[0, 4, 5]] == -1)   # zero direction, tmin > tmax, negative tmax
    s.close()


def test_degenerate_triangles_never_hit(ctx):
    tris = np.array([[0, 0, 0, 1, 1, 1, 2, 2, 2], [0, 0, 0, 0, 0, 0, 0, 0, 0],
                     [0.5, 0.5, 0.5, 0.5, 0.5, 0.5, 1, 0, 0]], np.float32)
    s = ctx.scene(soup_scene(tris))
    org, dirs = scenes.incoherent_rays(4000, seed=9, lo=-0.5, hi=2.5)
    h = s.trace_closest(org, dirs)
    assert np.all(h["id"] == -1)
    s.close()


def test_coincident_triangles_resolve_to_lowest_id(ctx):
    base = scenes.triangle_soup(300, seed=4, sigma=0.05)
    dup = np.concatenate([base, base[::-1], base], 0)   # every triangle three times
    s = ctx.scene(soup_scene(dup))
    org, dirs = scenes.incoherent_rays(8000, seed=6)
    h = s.trace_closest(org, dirs)
    assert_same(h, oracle.CpuBVH(dup).trace(org, dirs))
    assert (h["id"] >= 0).any()
    # base triangle k sits at ids k, 599 - k and 600 + k: the hit is always the first copy
    assert np.array_equal(h["id"], oracle.trace_brute(base, org, dirs)["id"])
    s.close()


def test_axis_aligned_rays(ctx):
    tris = scenes.triangle_soup(5000, seed=7, sigma=0.02)
    g = np.linspace(0.0, 1.0, 40, dtype=np.float32)
    X, Y = np.meshgrid(g, g)
    orgs, dirs = [], []
    for axis in range(3):
        for sign in (1.0, -1.0):
            o = np.zeros((X.size, 4), np.float32)
            a, b = [k for k in range(3) if k != axis]
            o[:, a], o[:, b] = X.ravel(), Y.ravel()
            o[:, axis] = -0.5 if sign > 0 else 1.5
            d = np.zeros((X.size, 4), np.float32)
            d[:, axis] = sign
            d[:, 3] = np.inf
            orgs.append(o)
            dirs.append(d)
    org, dirs = np.concatenate(orgs), np.concatenate(dirs)
    s = ctx.scene(soup_scene(tris))
    h = s.trace_closest(org, dirs)
    assert_same(h, oracle.trace_brute(tris, org, dirs))
    assert (h["id"] >= 0).mean() > 0.1
    s.close()


def test_tiny_images_and_depth_zero(ctx, orc_tables):
    sc = scenes.cornell(3, 2)
    for spp, depth in ((1, 0), (3, 1), (2, 8)):
        p = scenes.render_params(spp, depth, fb.FL_SPECTRAL_BINS60)
        s = ctx.scene(sc)
        xyz = np.zeros((2, 3, 3), np.float64)
        _, st = s.render(p, film_xyz64=xyz)
        s.close()
        cpu, cnt = oracle.render(sc, orc_tables, p)
        assert st["paths"] == cnt["paths"] == 6 * spp
        assert np.allclose(xyz, cpu, rtol=1e-4, atol=1e-7)


def test_scene_without_lights_renders_black(ctx):
    sc = scenes.cornell(16, 16)
    dark = scenes.Scene(sc.verts, sc.tri_material, sc.materials, [], sc.camera)
    s = ctx.scene(dark)
    rgb, st = s.render(scenes.render_params(4, 8, fb.FL_SPECTRAL_HERO4))
    s.close()
    assert st["paths"] == 16 * 16 * 4
    assert np.all(rgb == 0.0)
