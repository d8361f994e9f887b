"""The guiding oracle's analytic gradient (forward, vMF mixture head, back-propagation)
against central finite differences of its loss, with FP16 rounding switched off."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
import guide_records as gr  # noqa: E402

LAYER = [(0, 5120), (5120, 9216), (9216, 13312), (13312, 17408), (17408, 20032)]


@pytest.mark.parametrize("learned", [False, True])
def test_gradient_matches_finite_differences(learned):
    """learned: the loss of the one-sample MIS density c q + (1 - c) p_bsdf, whose gradient
    also reaches the selection output (head row 40, the last 64 weights)"""
    rec = gr.records(64, seed=3)
    w = gr.weights(seed=4).astype(np.float64)
    oracle.guide_set_exact(True)
    try:
        g, loss = oracle.guide_gradient(w.astype(np.float32), rec, gr.BMIN, gr.BMAX, learned)
        if learned:
            assert np.abs(g[-64:]).max() > 0
        else:
            assert np.all(g[-64:] == 0)
        assert np.isfinite(loss) and loss != 0.0
        rng = np.random.default_rng(5)
        for lo, hi in LAYER:
            # the largest gradient entries of each layer plus a few random ones
            idx = list(np.argsort(-np.abs(g[lo:hi]))[:4] + lo) + list(rng.integers(lo, hi, 4))
            for i in idx:
                h = 1e-3 * max(1.0, abs(w[i]))
                wp = w.copy()
                wp[i] += h
                wm = w.copy()
                wm[i] -= h
                _, lp = oracle.guide_gradient(wp.astype(np.float32), rec, gr.BMIN, gr.BMAX, learned)
                _, lm = oracle.guide_gradient(wm.astype(np.float32), rec, gr.BMIN, gr.BMAX, learned)
                fd = (lp - lm) / (2 * h)
                assert abs(fd - g[i]) <= 2e-2 * max(abs(g[i]), 1e-2 * np.abs(g[lo:hi]).max()) + 1e-4, (i, fd, g[i])
    finally:
        oracle.guide_set_exact(False)


def test_mixture_is_normalised():
    rec = gr.records(32, seed=6)
    m = oracle.guide_eval(gr.weights(seed=7), rec, gr.BMIN, gr.BMAX)
    assert np.allclose(m[:, :8].sum(axis=1), 1.0, atol=1e-5)
    mu = m[:, 8:32].reshape(-1, 8, 3)
    assert np.allclose(np.linalg.norm(mu, axis=2), 1.0, atol=1e-5)
    assert np.all(m[:, 32:40] >= np.exp(-2.0) * 0.999) and np.all(m[:, 32:40] <= np.exp(7.0) * 1.001)
    assert np.all((m[:, 40] >= 0.2) & (m[:, 40] <= 0.7))
