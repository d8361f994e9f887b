"""Learned path guiding on the GPU: the tensor-core forward pass and training gradient
against the CPU oracle, the guided renderer without guiding against fl_render, the
unbiasedness of the one-sample MIS estimator with an untrained network, and what the
trained network gains on the caustic scene at equal samples per pixel."""
import numpy as np
import pytest

import filianore_b200 as fb
import guide_records as gr
import oracle
from filianore_b200 import scenes

pytestmark = pytest.mark.gpu

LAYER = [(0, 5120), (5120, 9216), (9216, 13312), (13312, 17408), (17408, 20032)]


@pytest.fixture(scope="module")
def ctx():
    c = fb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("kernel", [fb.FL_GUIDE_TRAIN_MMA_SYNC, fb.FL_GUIDE_TRAIN_TCGEN05])
@pytest.mark.parametrize("learned", [False, True])
def test_gradient_matches_oracle(ctx, learned, kernel):
    """FP16 tensor-core forward + backward against the oracle (same FP16 roundings, double
    accumulation), on the mma.sync training kernel and on the tcgen05 one: relative L2 error
    of every layer's gradient below 1e-2; with the learned selection probability, the loss of
    the one-sample MIS density as well."""
    g = fb.Guide(ctx, max_records=8192, batch=1024, learn_select=learned, train_kernel=kernel)
    w = gr.weights(seed=11)
    g.set_weights(w)
    rec = gr.records(3000, seed=12)
    gg, lg = g.gradient(rec, gr.BMIN, gr.BMAX)
    gc, lc = oracle.guide_gradient(w, rec, gr.BMIN, gr.BMAX, learned)
    assert np.isfinite(gg).all()
    assert abs(lg / lc - 1) < 1e-3, (lg, lc)
    for lo, hi in LAYER:
        err = np.linalg.norm(gg[lo:hi] - gc[lo:hi]) / np.linalg.norm(gc[lo:hi])
        assert err < 1e-2, (lo, err)
    g.close()


def test_mixture_matches_oracle(ctx):
    g = fb.Guide(ctx, max_records=8192, batch=1024)
    w = gr.weights(seed=13)
    g.set_weights(w)
    rec = gr.records(1000, seed=14)
    mg = g.eval(rec, gr.BMIN, gr.BMAX)
    mc = oracle.guide_eval(w, rec, gr.BMIN, gr.BMAX)
    assert np.abs(mg[:, :32] - mc[:, :32]).max() < 5e-3
    assert np.abs(mg[:, 32:40] / mc[:, 32:40] - 1).max() < 5e-3
    assert np.abs(mg[:, 40] - mc[:, 40]).max() < 5e-3  # selection probability
    g.close()


def test_unguided_pass_equals_plain_render(ctx):
    """With guiding off (no sampling, no training) the guided wave loop draws the same
    random numbers and takes the same paths as fl_render."""
    sc = scenes.cornell(48, 48)
    s = ctx.scene(sc)
    p = scenes.render_params(8, 8, fb.FL_SPECTRAL_HERO4)
    a = np.zeros((48, 48, 3), np.float64)
    b = np.zeros((48, 48, 3), np.float64)
    s.render(p, film_xyz64=a)
    g = fb.Guide(ctx)
    g.render(s, p, 0, film_xyz64=b)
    assert np.array_equal(a, b)
    g.close()
    s.close()


@pytest.mark.parametrize("learn_select", [False, True])
def test_untrained_guide_is_unbiased(ctx, learn_select):
    """One-sample MIS with an arbitrary (untrained) mixture, and with c fixed or taken per
    point from the network: the image converges to the plain render's. 1024 spp; tolerances
    are several standard errors."""
    sc = scenes.cornell(32, 32)
    s = ctx.scene(sc)
    p = scenes.render_params(1024, 8, fb.FL_SPECTRAL_HERO4)
    plain = np.zeros((32, 32, 3), np.float64)
    s.render(p, film_xyz64=plain)
    g = fb.Guide(ctx, seed=3, select_prob=0.5, learn_select=learn_select)
    guided = np.zeros((32, 32, 3), np.float64)
    g.render(s, scenes.render_params(1024, 8, fb.FL_SPECTRAL_HERO4, sample_offset=5000), fb.FL_GUIDE_SAMPLE,
             film_xyz64=guided)
    assert abs(guided.mean() / plain.mean() - 1) < 1.5e-2
    bp = plain.reshape(4, 8, 4, 8, 3).mean(axis=(1, 3))
    bg = guided.reshape(4, 8, 4, 8, 3).mean(axis=(1, 3))
    assert np.all(np.abs(bg / bp - 1) < 6e-2), np.abs(bg / bp - 1).max()
    g.close()
    s.close()


def test_trained_guide_lowers_caustic_error(ctx):
    """Caustic scene (glass sphere under a tiny, bright sphere light), 256 x 256: after online
    training (48 passes of 4 spp; Adam lr 1e-3, batches of 32 K records; rendering with the
    weight average), the guided render's mean squared error against a 4096-spp plain render
    is below the plain render's at the same 64 samples per pixel: below 0.85 x over the image
    and 0.75 x in the caustic (the brightest 3% of the reference). Errors are averaged over
    six renders per estimator, and the guided one over two independently trained guides:
    training order varies from run to run (atomics). Six single guides measured 0.48-0.67 x
    over the image and 0.43-0.57 x in the caustic."""
    R = 256
    sc = scenes.caustic(R, R, slices=128, stacks=65)
    s = ctx.scene(sc)
    ref = np.zeros((R, R, 3), np.float64)
    s.render(scenes.render_params(4096, 8, fb.FL_SPECTRAL_HERO4, sample_offset=1 << 20), film_xyz64=ref)
    ref /= 4096
    caustic = ref[..., 1] >= np.quantile(ref[..., 1], 0.97)

    def mean_mse(render):
        full, region = [], []
        for k in range(6):
            img = np.zeros((R, R, 3), np.float64)
            render(img, 7000 + 64 * k)
            d = (img / 64 - ref) ** 2
            full.append(d.mean())
            region.append(d[caustic].mean())
        return np.array([np.mean(full), np.mean(region)])
    e_plain = mean_mse(lambda f, off: s.render(scenes.render_params(64, 8, fb.FL_SPECTRAL_HERO4, sample_offset=off),
                                               film_xyz64=f))
    e_guided = []
    for seed in (5, 6):
        g = fb.Guide(ctx, seed=seed, learning_rate=1e-3, select_prob=0.5, batch=32768, max_records=1 << 19,
                     steps_per_wave=32, weight_average=0.99)
        for k in range(48):
            flags = fb.FL_GUIDE_TRAIN | (fb.FL_GUIDE_SAMPLE if k > 0 else 0)
            g.render(s, scenes.render_params(4, 8, fb.FL_SPECTRAL_HERO4, sample_offset=(1 << 16) + 4 * k), flags)
        assert g.info()["adam_steps"] > 0
        e_guided.append(mean_mse(lambda f, off: g.render(
            s, scenes.render_params(64, 8, fb.FL_SPECTRAL_HERO4, sample_offset=off), fb.FL_GUIDE_SAMPLE, film_xyz64=f)))
        g.close()
    ratio = np.mean(e_guided, axis=0) / e_plain
    assert ratio[0] < 0.85 and ratio[1] < 0.75, (ratio, e_guided, e_plain)
    s.close()


def test_guide_config_is_validated(ctx):
    for bad in ({"weight_average": 1.0}, {"weight_average": -0.1}, {"batch": 100}, {"select_prob": 1.0},
                {"learn_select": 2}):
        with pytest.raises(fb.FlError):
            fb.Guide(ctx, **bad)
