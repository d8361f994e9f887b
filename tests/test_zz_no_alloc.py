"""fl_render_noalloc, the render entry point for callers that cannot allocate device memory
at render time (their device memory is owned and budgeted by a host application, or an
allocation would synchronise the device). It keeps its path state in a fixed device array
inside the library instead of allocating. Checked through the C ABI against fl_render on
two calls in a row (the second call must not see anything the first one left in the shared
array), and, on the second call, that the device's free memory is the same before and after
the call. This file is collected last so that a stop at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

import filianore_b200 as fb
from filianore_b200 import scenes

pytestmark = pytest.mark.gpu


def _films(sc):
    import torch
    W, H = sc.camera["width"], sc.camera["height"]
    return (torch.zeros((H, W, 3), dtype=torch.float32, device="cuda"),
            torch.zeros((H, W, 3), dtype=torch.float64, device="cuda"))


def _noalloc(scene_h, sc, params, films):
    """One fl_render_noalloc call into the caller's device films; returns the device free
    memory (cudaMemGetInfo) just before and just after the call, and the stats."""
    import torch
    rgb, xyz = films
    xyz.fill_(7.0)  # must be cleared by the call
    torch.cuda.synchronize()
    stats = fb.fl_render_stats()
    cam = sc.camera_struct()
    free_before = torch.cuda.mem_get_info()[0]
    fb.check(fb.lib().fl_render_noalloc(scene_h.h, C.byref(cam), C.byref(params), C.c_void_p(rgb.data_ptr()),
                                        C.c_void_p(xyz.data_ptr()), C.byref(stats)), scene_h.ctx.h)
    free_after = torch.cuda.mem_get_info()[0]
    return free_before, free_after, stats


@pytest.mark.parametrize("variant,mode", [("materials", fb.FL_SPECTRAL_HERO4), ("lambert", fb.FL_SPECTRAL_BINS60)])
def test_noalloc_render_matches_fl_render(variant, mode):
    ctx = fb.Context(0)
    sc = scenes.cornell(96, 80, variant)
    s = ctx.scene(sc)
    p = scenes.render_params(8, 8, mode)
    want_xyz = np.zeros((80, 96, 3), np.float64)
    want_rgb, want_stats = s.render(p, film_xyz64=want_xyz)
    films = _films(sc)
    for call in range(2):
        free_before, free_after, stats = _noalloc(s, sc, p, films)
        if call == 1:
            # the defining property: after the first call on the device (which looks the
            # fixed array up), a call takes no device memory at all
            assert free_after == free_before
        assert stats.paths == want_stats["paths"] and stats.traversal_errors == 0
        rgb, xyz = (f.cpu().numpy() for f in films)
        # identical per-sample streams; only the FP64 summation order of the film differs
        np.testing.assert_allclose(xyz, want_xyz, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(rgb, want_rgb, rtol=1e-5, atol=1e-6)
    s.close()
    ctx.close()


def test_noalloc_render_large_frame_spans_several_waves():
    """a frame larger than one fixed-size wave gives the same image as fl_render"""
    ctx = fb.Context(0)
    sc = scenes.procedural_spheres(n_spheres=8, slices=32, stacks=17, width=320, height=240, extent=4.0,
                                   sphere_light=(0.0, 4.0, 0.0, 0.5, 40.0))
    s = ctx.scene(sc)
    p = scenes.render_params(4, 8, fb.FL_SPECTRAL_HERO4)
    want_xyz = np.zeros((240, 320, 3), np.float64)
    s.render(p, film_xyz64=want_xyz)
    films = _films(sc)
    for call in range(2):
        free_before, free_after, stats = _noalloc(s, sc, p, films)
        if call == 1:
            assert free_after == free_before
        assert stats.paths == 320 * 240 * 4
        np.testing.assert_allclose(films[1].cpu().numpy(), want_xyz, rtol=1e-9, atol=1e-12)
    s.close()
    ctx.close()
