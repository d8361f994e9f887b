"""Corrected GGX mode (FL_RENDER_CORRECTED_GGX): the density of the visible normals the
sampler draws, sampled on wo's side, instead of the reference's D |cos| with upper-hemisphere
sampling (quirks Q1, Q2). The GPU against the oracle in that mode, and a white-furnace check
of the estimator itself: a rough conductor plane under a constant environment shows its
directional albedo, which the oracle's BSDF gives by quadrature independently of any
sampling density."""
import numpy as np
import pytest

import filianore_b200 as fb
import oracle
from filianore_b200 import scenes
from filianore_b200 import types as T

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fb.Context(0)
    yield c
    c.close()


def render_xyz(ctx, sc, p):
    s = ctx.scene(sc)
    xyz = np.zeros((sc.camera["height"], sc.camera["width"], 3), np.float64)
    _, st = s.render(p, film_xyz64=xyz)
    s.close()
    return xyz, st


@pytest.mark.parametrize("variant", ["materials", "glass"])
def test_corrected_mode_matches_oracle(ctx, orc_tables, variant):
    sc = scenes.cornell(48, 48, variant=variant)
    p = scenes.render_params(4, 8, fb.FL_SPECTRAL_BINS60, flags=fb.FL_RENDER_CORRECTED_GGX)
    xyz, _ = render_xyz(ctx, sc, p)
    cpu, _ = oracle.render(sc, orc_tables, p)
    close = np.all(np.abs(xyz - cpu) <= np.maximum(1e-4 * np.abs(cpu), 1e-6), axis=-1).mean()
    assert close >= 0.99
    assert abs(xyz.mean() / cpu.mean() - 1) < 2e-3
    # and the mode changes the image (the rough lobes are sampled differently)
    ref_mode, _ = render_xyz(ctx, sc, scenes.render_params(4, 8, fb.FL_SPECTRAL_BINS60))
    assert not np.array_equal(ref_mode, xyz)


def furnace_albedo(material, theta_o, n_theta=512, n_phi=1024):
    th = (np.arange(n_theta) + 0.5) * (np.pi / 2) / n_theta
    ph = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    wi = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1).reshape(-1, 3)
    wo = np.array([np.sin(theta_o), 0.0, np.cos(theta_o)])
    fc = oracle.bsdf_fcos(material, wo, wi).reshape(n_theta, n_phi)
    return float(np.sum(fc * np.sin(TH)) * (np.pi / 2 / n_theta) * (2 * np.pi / n_phi))


def test_furnace_conductor_albedo(ctx):
    mat = {"type": fb.FL_MAT_CONDUCTOR, "rgb": (1.0, 1.0, 1.0), "roughness": 0.5, "eta": 0.2, "k": 3.9}
    big = 1000.0
    plane = np.array([[-big, 0, -big, -big, 0, big, big, 0, big], [-big, 0, -big, big, 0, big, big, 0, -big]],
                     np.float32)
    env = [{"type": fb.FL_LIGHT_ENV, "radiance": 1.0}]
    cam = {"position": (0.0, 1.0, -1.0), "look_at": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "vfov": 0.5,
           "width": 8, "height": 8}
    sky_cam = {"position": (0.0, 1.0, 0.0), "look_at": (0.0, 2.0, 0.0), "up": (0.0, 0.0, 1.0), "vfov": 0.5,
               "width": 8, "height": 8}
    sc = scenes.Scene(plane, np.zeros(2, np.uint32), [mat], env, cam)
    sky = scenes.Scene(plane, np.zeros(2, np.uint32), [mat], env, sky_cam)
    spp = 8192
    y_sky = render_xyz(ctx, sky, scenes.render_params(16, 4, fb.FL_SPECTRAL_BINS60))[0][..., 1].mean() / 16
    m = T.fl_material()
    m.type, m.roughness, m.eta, m.k = mat["type"], mat["roughness"], mat["eta"], mat["k"]
    m.rgb[:] = [1.0, 1.0, 1.0]
    truth = furnace_albedo(m, np.pi / 4)
    p = scenes.render_params(spp, 4, fb.FL_SPECTRAL_BINS60, flags=fb.FL_RENDER_CORRECTED_GGX)
    corrected = render_xyz(ctx, sc, p)[0][..., 1].mean() / spp / y_sky
    reference = render_xyz(ctx, sc, scenes.render_params(spp, 4, fb.FL_SPECTRAL_BINS60))[0][..., 1].mean() / spp / y_sky
    print(f"furnace albedo: quadrature {truth:.5f} corrected {corrected:.5f} reference mode {reference:.5f}")
    assert abs(corrected / truth - 1) < 0.015
