"""Seeded synthetic inputs of the benchmark configurations (no dataset is involved).

* ``log_conductivity(x, seed, sigma)``: ``m(x) = sum_{j=1..32} a_j cos(2 pi w_j.x + phi_j)``
  with ``a_j ~ N(0, sigma^2)``, ``w_j`` integer in ``[-4, 4]^3``, ``phi_j ~ U[0, 2 pi)``;
  nodally interpolated into Q2 by ``Q2Space.project``.
* ``interior_points(n, seed)``: uniform random points strictly inside the unit box.
* ``vertical_lines(nlines, ndepth, seed)``: observation lines at random (x, y).
* ``normal_vector(ndof, seed)``: ``v ~ N(0, 1)``.
"""

import numpy as np


def field_params(seed=0, sigma=0.1, nterms=32):
    rng = np.random.default_rng(seed)
    a = rng.normal(0.0, sigma, nterms)
    w = rng.integers(-4, 5, size=(nterms, 3))
    phi = rng.uniform(0.0, 2.0 * np.pi, nterms)
    return a, w, phi


def log_conductivity(x, seed=0, sigma=0.1, nterms=32):
    a, w, phi = field_params(seed, sigma, nterms)
    x = np.asarray(x, dtype=np.float64)
    return np.cos(2.0 * np.pi * (x @ w.T) + phi[None, :]) @ a


def interior_points(n, seed=2, margin=0.05):
    rng = np.random.default_rng(seed)
    return margin + (1.0 - 2.0 * margin) * rng.random((n, 3))


def vertical_lines(nlines=60, ndepth=64, seed=3, margin=0.05):
    rng = np.random.default_rng(seed)
    xy = margin + (1.0 - 2.0 * margin) * rng.random((nlines, 2))
    z = np.linspace(margin, 1.0 - margin, ndepth)
    pts = np.concatenate([np.column_stack([np.repeat(xy[:, 0:1], ndepth, 1).ravel(),
                                           np.repeat(xy[:, 1:2], ndepth, 1).ravel(),
                                           np.tile(z, nlines)])])
    return pts


def normal_vector(ndof, seed=4):
    return np.random.default_rng(seed).standard_normal(ndof)
