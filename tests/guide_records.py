"""Seeded synthetic training records and weights for the path-guiding tests."""
import numpy as np

BMIN = np.array([-1.0, 0.0, -2.0], np.float32)
BMAX = np.array([3.0, 2.0, 2.0], np.float32)


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def records(n, seed=0):
    """(n, 20) records: points in the bounds, unit normals, wavelengths, directions mostly in
    the normal's hemisphere, densities, and heavy-tailed incident radiance (some zero)."""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 20), np.float32)
    r[:, 0:3] = BMIN + (BMAX - BMIN) * rng.random((n, 3))
    nrm = unit(rng.normal(size=(n, 3)))
    r[:, 3:6] = nrm
    r[:, 6] = 380.0 + 340.0 * rng.random(n)
    d = unit(rng.normal(size=(n, 3)))
    flip = np.sum(d * nrm, axis=1) < 0
    d[flip & (rng.random(n) < 0.9)] *= -1.0
    r[:, 7:10] = d
    r[:, 10] = 0.05 + rng.random(n)
    li = np.exp(rng.normal(0.0, 1.5, n))
    li[rng.random(n) < 0.2] = 0.0
    r[:, 11] = li
    return r


def weights(seed=0, scale=1.0):
    """He-uniform hidden layers, Xavier head (the guide's own initialisation scheme)"""
    rng = np.random.default_rng(seed)
    shapes = [(64, 80), (64, 64), (64, 64), (64, 64), (41, 64)]
    out = []
    for l, (o, i) in enumerate(shapes):
        lim = np.sqrt(6.0 / i) if l < 4 else np.sqrt(6.0 / (i + o))
        out.append((rng.uniform(-lim, lim, o * i) * scale).astype(np.float32))
    return np.concatenate(out)
