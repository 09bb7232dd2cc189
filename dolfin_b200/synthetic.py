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


def batched_square_meshes(count, seed, n_lo=8, n_hi=256, jitter=0.2):
    """Member specs of the batched workload: UnitSquareMesh(n, n), n drawn
    log-uniform in [n_lo, n_hi], interior vertices jittered by +-jitter*h,
    Lagrange degree 1 or 2, kappa uniform [0.5, 2] per vertex -- each member
    from its own seeded stream.  Returns a list of dicts (n, degree, seed)."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=count))).astype(int)
    degs = rng.integers(1, 3, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [dict(n=int(n), degree=int(d), seed=int(s), jitter=jitter) for n, d, s in zip(ns, degs, seeds)]


def build_batch_member(spec):
    """Engine objects of one batched member: (mesh, V, kappa Function, coords, kappa values)."""
    from . import FunctionSpace, Function, UnitSquareMesh
    n = spec["n"]
    mesh = UnitSquareMesh(n, n)
    x = jitter_interior(mesh.coordinates(), n, spec["jitter"], spec["seed"])
    mesh.set_coordinates(x)
    V = FunctionSpace(mesh, "Lagrange", spec["degree"])
    W = V if spec["degree"] == 1 else FunctionSpace(mesh, "Lagrange", 1)
    kv = uniform_field(mesh.num_vertices(), 0.5, 2.0, spec["seed"] + 1)
    return mesh, V, Function(W, kv), x, kv
