"""Parity of the scene features the reference has no class for (environment light,
analytic sphere light) together with every material, on procedural scenes: the GPU
renderer against the CPU oracle with the same per-pixel PCG32 streams, plus an
equal-spp MSE comparison against an FP64-accumulated high-spp oracle render."""
import numpy as np
import pytest

import filianore_b200 as fb
import oracle
from filianore_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fb.Context(0)
    yield c
    c.close()


def gpu_xyz(ctx, sc, p):
    s = ctx.scene(sc)
    xyz = np.zeros((sc.camera["height"], sc.camera["width"], 3), np.float64)
    _, stats = s.render(p, film_xyz64=xyz)
    s.close()
    return xyz, stats


def close_fraction(a, b, rtol, atol):
    return np.all(np.abs(a - b) <= np.maximum(rtol * np.abs(b), atol), axis=-1).mean()


def small_procedural():
    return scenes.procedural_spheres(n_spheres=12, slices=24, stacks=13, width=96, height=54, extent=4.0,
                                     sphere_light=(0.0, 4.0, 0.0, 0.5, 40.0))


# Measured on a B200: hero 99.85% of pixels within 1e-3 (99.69% within 1e-4), 60 bins 100%
# within 1e-4. The hero build contracts into FMAs and evaluates sin / cos in single
# precision, so a path can rarely take another discrete decision.
@pytest.mark.parametrize("mode,rtol,frac_min", [(fb.FL_SPECTRAL_HERO4, 1e-3, 0.995), (fb.FL_SPECTRAL_BINS60, 1e-4, 0.999)])
def test_procedural_scene_matches_oracle(ctx, orc_tables, mode, rtol, frac_min):
    sc = small_procedural()
    p = scenes.render_params(4, 8, mode)
    xyz, stats = gpu_xyz(ctx, sc, p)
    cpu, cnt = oracle.render(sc, orc_tables, p)
    assert stats["paths"] == cnt["paths"] and stats["traversal_errors"] == 0
    assert close_fraction(xyz, cpu, rtol, 1e-5) >= frac_min
    assert abs(xyz.mean() / cpu.mean() - 1) < 1e-2


def test_caustic_scene_matches_oracle(ctx, orc_tables):
    """Glass sphere + tiny sphere light: per pixel in the 60-bin parity build (no FMA,
    correctly rounded sin/cos), >= 99% of pixels within 1e-4. The hero build contracts into
    FMAs, which the long specular chains turn into different paths in some pixels, so its
    per-pixel bound has two parts: >= 88% of pixels within 1e-3 relative (91.0% measured),
    and the per-pixel differences of the rest no larger than Monte Carlo noise: their 99th
    percentile at most a quarter of the 99th percentile of the difference between two oracle
    renders with independent samples (0.12 of it measured), their maximum below the noise's
    maximum; the image mean within 1e-2."""
    sc = scenes.caustic(64, 64, slices=32, stacks=17)
    p = scenes.render_params(8, 8, fb.FL_SPECTRAL_BINS60)
    xyz, _ = gpu_xyz(ctx, sc, p)
    cpu, _ = oracle.render(sc, orc_tables, p)
    assert close_fraction(xyz, cpu, 1e-4, 1e-6) >= 0.99
    p = scenes.render_params(16, 8, fb.FL_SPECTRAL_HERO4)
    xyz, _ = gpu_xyz(ctx, sc, p)
    cpu, _ = oracle.render(sc, orc_tables, p)
    cpu2, _ = oracle.render(sc, orc_tables, scenes.render_params(16, 8, fb.FL_SPECTRAL_HERO4, sample_offset=1000))
    assert close_fraction(xyz, cpu, 1e-3, 1e-5) >= 0.88
    diff = np.abs(xyz - cpu).max(axis=-1)
    noise = np.abs(cpu2 - cpu).max(axis=-1)
    assert np.quantile(diff, 0.99) <= 0.25 * np.quantile(noise, 0.99), (np.quantile(diff, 0.99), np.quantile(noise, 0.99))
    assert diff.max() <= noise.max()
    assert abs(xyz.mean() / cpu.mean() - 1) < 1e-2


def test_equal_spp_mse_matches_oracle(ctx, orc_tables):
    """At equal spp the GPU image's MSE against a 512-spp FP64 oracle render is
    statistically indistinguishable from the oracle's own (independent sample indices)."""
    sc = scenes.procedural_spheres(n_spheres=6, slices=16, stacks=9, width=32, height=18, extent=3.0,
                                   sphere_light=(0.0, 3.0, 0.0, 0.5, 40.0))
    gt, _ = oracle.render(sc, orc_tables, scenes.render_params(512, 8, fb.FL_SPECTRAL_HERO4, sample_offset=100000))
    gt /= 512
    mses_gpu, mses_cpu = [], []
    for k in range(4):
        g, _ = gpu_xyz(ctx, sc, scenes.render_params(16, 8, fb.FL_SPECTRAL_HERO4, sample_offset=1000 + 16 * k))
        c, _ = oracle.render(sc, orc_tables, scenes.render_params(16, 8, fb.FL_SPECTRAL_HERO4, sample_offset=5000 + 16 * k))
        mses_gpu.append(np.mean((g / 16 - gt) ** 2))
        mses_cpu.append(np.mean((c / 16 - gt) ** 2))
    ratio = np.mean(mses_gpu) / np.mean(mses_cpu)
    assert 0.6 < ratio < 1.6, (mses_gpu, mses_cpu)
