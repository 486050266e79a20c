"""Shared test helpers: small seeded problems and their oracle/product forms."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

from pefdtd import workloads  # noqa: E402


def small_spec(shape=(24, 28, 32), h=0.4e-3, n_grains=12, seed=5, nt=120, sponge=4,
               fabric=("watson", 30.0, 5.0)):
    nz, ny, nx = shape
    d = (min(ny, nx) - 6) * h
    return dict(shape=shape, h=h, diameter=d, height=(nz - 8) * h, n_grains=n_grains,
                fabric=fabric, f0=1.0e6 * 0.2e-3 / h, n_cycles=3, nt=nt, sponge=sponge,
                aperture=d / 3, seed=seed)


def make_small(nt=120, **kw):
    return workloads.make_problem(small_spec(nt=nt, **kw), use_gpu=False)


def oracle_prob(p, **kw):
    from oracle.oracle import problem_from_workload
    return problem_from_workload(p, **kw)


def rel_l2(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def synthetic_echo(nt, dt, f0):
    """A deterministic stand-in trace for sweep-protocol tests: a Gaussian
    burst at the 2 x 100 mm first-echo time plus a weak later coda."""
    t = np.arange(int(nt)) * float(dt)
    t1 = 0.200 / 3850.0
    burst = np.sin(2 * np.pi * f0 * (t - t1)) * np.exp(-((t - t1) * f0 / 1.5) ** 2)
    coda = 0.05 * np.sin(2 * np.pi * 0.7 * f0 * t) * np.exp(-((t - 30e-6) / 8e-6) ** 2)
    return (burst + coda).astype(np.float32)
