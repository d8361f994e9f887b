"""The oracle's closest-hit semantics: its BVH agrees with brute force (watertight test,
lowest id on ties), including edge cases."""
import numpy as np

import oracle
from filianore_b200 import scenes


def _same(a, b):
    assert np.array_equal(a["id"], b["id"])
    hit = a["id"] >= 0
    assert np.array_equal(a["t"][hit], b["t"][hit])
    assert np.array_equal(a["u"][hit], b["u"][hit])
    assert np.array_equal(a["v"][hit], b["v"][hit])


def test_bvh_equals_brute_force_soup():
    tris = scenes.triangle_soup(4000, seed=3, sigma=0.02)
    org, dirs = scenes.incoherent_rays(3000, seed=4)
    bvh = oracle.CpuBVH(tris)
    _same(bvh.trace(org, dirs), oracle.trace_brute(tris, org, dirs))


def test_bvh_equals_brute_force_cornell():
    sc = scenes.cornell(32, 32)
    org, dirs = scenes.incoherent_rays(5000, seed=5, lo=0.01, hi=0.99)
    _same(oracle.CpuBVH(sc.verts).trace(org, dirs), oracle.trace_brute(sc.verts, org, dirs))


def test_shared_edges_are_watertight():
    """rays through the shared diagonal of a quad split into two triangles hit exactly one
    of them (no leaks); ties on the edge resolve to the lower id"""
    quad = np.array([[0, 0, 0, 1, 0, 0, 1, 1, 0], [0, 0, 0, 1, 1, 0, 0, 1, 0]], np.float32)
    s = np.linspace(0.001, 0.999, 997, dtype=np.float32)
    org = np.stack([s, s, np.full_like(s, -1), np.zeros_like(s)], 1).astype(np.float32)
    dirs = np.tile(np.array([0, 0, 1, np.inf], np.float32), (s.size, 1))
    h = oracle.CpuBVH(quad).trace(org, dirs)
    assert np.all(h["id"] >= 0)
    assert np.all(h["id"] == 0)   # both triangles contain the diagonal: lower id wins
    assert np.all(h["t"] == 1.0)


def test_tmin_tmax_are_exclusive():
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    org = np.array([[0.2, 0.2, -1, 0], [0.2, 0.2, -1, 1.0], [0.2, 0.2, -1, 0]], np.float32)
    dirs = np.array([[0, 0, 1, 1.0], [0, 0, 1, np.inf], [0, 0, 1, 1.0000001]], np.float32)
    h = oracle.CpuBVH(tri).trace(org, dirs)
    assert list(h["id"]) == [-1, -1, 0]


def test_empty_scene_and_degenerate_rays():
    tris = np.zeros((0, 9), np.float32)
    org, dirs = scenes.incoherent_rays(10)
    h = oracle.CpuBVH(tris).trace(org, dirs)
    assert np.all(h["id"] == -1)
    one = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    zero_dir = np.zeros((1, 4), np.float32)
    zero_dir[0, 3] = np.inf
    h = oracle.CpuBVH(one).trace(np.array([[0.2, 0.2, -1, 0]], np.float32), zero_dir)
    assert h["id"][0] == -1


def test_degenerate_triangles_never_hit():
    tris = np.array([[0, 0, 0, 1, 1, 1, 2, 2, 2], [0, 0, 0, 0, 0, 0, 0, 0, 0]], np.float32)
    org, dirs = scenes.incoherent_rays(2000, seed=9, lo=-0.5, hi=2.5)
    h = oracle.trace_brute(tris, org, dirs)
    assert np.all(h["id"] == -1)
