"""Pins of the CPU oracle (test infrastructure) against the reference.

(a) bit for bit against the reference's own label-path and dense kernels,
    compiled for the host from the reference sources (oracle/_ref);
(b) against golden traces of the reference's NumPy array path, FP64 on the
    CPU and FP32 through a NumPy stand-in for CuPy (tests/golden).
"""
import os

import numpy as np
import pytest

from helpers import make_small, oracle_prob, rel_l2
from oracle import oracle as O
from pefdtd import damping

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(O.ref_lib() is None, reason="reference harness not built")


@needs_ref
@pytest.mark.parametrize("record", ["pressure", "vz", "vx"])
@pytest.mark.parametrize("order", [8, 6, 2])
def test_oracle_bit_exact_vs_reference_label_kernels(record, order):
    p = make_small(nt=90, shape=(21, 26, 29), n_grains=9, sponge=3)
    from pefdtd.coeffs import optimised_coeffs, taylor_coeffs
    p["coeffs"] = optimised_coeffs(order) if order > 2 else taylor_coeffs(2)
    pr = oracle_prob(p, record=record, damped_record=False)
    a = O.run_oracle(pr, fma_mode=0)
    b = O.run_reference_labels(pr, slab=5)
    assert np.abs(b).max() > 0
    assert np.array_equal(a, b)


@needs_ref
def test_oracle_bit_exact_with_fluid_mask_and_odd_grid():
    p = make_small(nt=80, shape=(17, 23, 19), n_grains=6, sponge=2)
    mask = damping.fluid_damp_mask(p["lab"], 0.05)
    pr = oracle_prob(p, record="pressure", damped_record=False, damp_mask=mask)
    a, sa = O.run_oracle(pr, fma_mode=0, return_state=True)
    b, sb = O.run_reference_labels(pr, slab=32, return_state=True)
    assert np.array_equal(a, b)
    assert np.array_equal(sa, sb)


@needs_ref
def test_reference_dense_equals_label_path_and_oracle_damped_record():
    # the reference's own --quick gate (sim/core/validate_labels.py:66-100),
    # and the dense path's end-of-step damped recording in the oracle
    p = make_small(nt=70, shape=(20, 24, 24), n_grains=7, sponge=6)
    pr = oracle_prob(p, record="pressure", damped_record=True)
    dense = O.run_reference_dense(pr)
    a = O.run_oracle(pr, fma_mode=0)
    assert np.array_equal(a, dense)
    pr_l = oracle_prob(p, record="vz", damped_record=False)
    assert np.array_equal(O.run_reference_labels(pr_l), O.run_reference_dense(pr_l))


@needs_ref
def test_oracle_many_materials_dense():
    # more than 254 materials: only the reference's dense kernels apply
    p = make_small(nt=40, shape=(20, 30, 30), n_grains=300, sponge=2)
    assert p["n_grains"] > 255
    pr = oracle_prob(p, record="vz", damped_record=True)
    assert np.array_equal(O.run_oracle(pr, fma_mode=0), O.run_reference_dense(pr))


def _golden_problem(g, record, dtype):
    from pefdtd.materials import material_tables
    lab = g["lab"].astype(np.int32)
    Ct, rho_t = material_tables(g["axes"])
    if dtype == np.float64:
        from pefdtd.fdtd import _material_tables64
        Ct, rho_t = _material_tables64(g["axes"], 1500.0, 300.0)
    pts = [tuple(q) for q in g["src"]]
    w = float(g["w"])
    p = dict(lab=lab, mats=(lab + 1), Ct=Ct, rho_t=rho_t, h=float(g["h"]), dt=float(g["dt"]),
             nt=int(g["nt"]), coeffs=g["coeffs"], wavelet=g["wavelet"], sponge=int(g["sponge"]),
             src_pts=[(q, w) for q in pts], rec_groups=[(pts, np.full(len(pts), w))],
             record=record)
    return oracle_prob(p, record=record, damped_record=True, dtype=dtype)


@pytest.mark.parametrize("record", ["pressure", "vz"])
def test_oracle_vs_reference_numpy_path_golden(record):
    g = np.load(os.path.join(GOLD, "forward_small.npz"))
    ref64 = g[f"{record}_f64"].ravel()
    ref32 = g[f"{record}_f32"].ravel()
    o64 = O.run_oracle(_golden_problem(g, record, np.float64), dtype=np.float64).ravel()
    o32 = O.run_oracle(_golden_problem(g, record, np.float32), dtype=np.float32).ravel()
    # same physics, different rounding order: the array path pre-scales the
    # taps by c/h and moves strains pairwise
    assert rel_l2(o64, ref64) < 1e-7
    assert rel_l2(o32, ref32) < 1e-5
    assert rel_l2(o32, ref64) < 1e-5
