"""Seeded synthetic inputs of the benchmark workloads: jittered unit meshes
and random nodal coefficient fields (numpy default_rng streams, host side)."""
from __future__ import annotations

import numpy as np


def jitter_interior(coords, n, amplitude, seed):
    """Move every interior vertex of a unit box mesh with n cells per side by
    an i.i.d. uniform offset in [-amplitude*h, amplitude*h]^d, h = 1/n.
    Boundary vertices stay put.  Returns a new array."""
    x = np.array(coords, np.float64, copy=True)
    h = 1.0 / n
    interior = np.all((x > 0.5 * h) & (x < 1.0 - 0.5 * h), axis=1)
    rng = np.random.default_rng(seed)
    delta = rng.uniform(-amplitude * h, amplitude * h, size=x.shape)
    x[interior] += delta[interior]
    return x


def uniform_field(n, lo, hi, seed):
    return np.random.default_rng(seed).uniform(lo, hi, size=n)


def lognormal_field(n, sigma, seed):
    """kappa = exp(g), g ~ N(0, sigma^2) i.i.d. per vertex."""
    return np.exp(np.random.default_rng(seed).normal(0.0, sigma, size=n))
