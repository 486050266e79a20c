"""Parity at the benchmark configurations' full lengths, where the echo is.

The bar: traces within relative L2 1e-5 of the reference's own update
kernels run on the same inputs, the Hilbert-envelope pick of the disk's
bottom-face echo identical, and the FP32 error against an FP64 run of the
same kernels stated.

* disk_small (64 x 96 x 96, 50 grains) at its full 2000 steps: bit-exact
  against the oracle, within 1e-5 of the reference's label-path kernels. Its
  20-cell sponge covers the probe and both disk faces (the disk is 50 of the
  64 planes), so the reference's sponge removes the bottom echo: after the
  transmitted burst the probe trace falls by more than ten orders of
  magnitude and stays there.
* the same disk with a 6-cell sponge, which leaves both faces outside it:
  the bottom-face echo comes back at 0.6 of the burst's envelope; full 2000
  steps against the reference's kernels and an FP64 run, echo pick identical
  and inside the echo window.
* disk_prod (160 x 256 x 256, 500 grains) over the first 1800 steps (burst
  and bottom echo) against the reference's dense kernels, whose trace is a
  fixture (tests/golden/make_disk_prod_echo.py; tens of minutes on the host).

The "reference's own update" is checked in both of its builds: the host
build (oracle/_ref/libref_cpu.so, every product rounded separately) and the
GPU build (oracle/_ref/libref_gpu.so: the reference's kernel strings compiled
by nvcc with default FMA contraction, as its NVRTC build runs them, launched
with its launch shapes). The GPU build makes the full 6000 steps of disk_prod
affordable, so that configuration is compared over its whole length.
"""
import os

import numpy as np
import pytest

from helpers import oracle_prob, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5
# "identical echo picks": the same sample index of the envelope maximum, and
# parabolically refined times within this fraction of a sample (disk_prod's
# FP32 traces against the reference's builds differ there by ~0.003 of a
# sample: rounding, not arrival)
PICK_REFINE_TOL = 1e-2
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "disk_prod_ref_echo.npz")


def _fwd(p, **kw):
    from pefdtd import fdtd
    return fdtd.forward_fused_labels(p["lab"], p["axes"], p["h"], p["dt"], p["nt"], p["src_pts"],
                                     p["wavelet"], p["rec_groups"], coeffs=p["coeffs"],
                                     sponge_width=p["sponge"], record="vz", damped_record=True, **kw)


def _echo_picks(p, *traces):
    from pefdtd import wavelets, workloads
    t = np.arange(p["nt"]) * p["dt"]
    t_lo, w_lo, w_hi = workloads.bottom_echo_window(p)
    picks = [wavelets.pick_peak(t, np.asarray(x, float).ravel(), t_lo=t_lo, dt=p["dt"]) for x in traces]
    return picks, t_lo, w_lo, w_hi


def test_disk_small_full_length_vs_oracle_and_reference():
    from pefdtd import workloads
    if O.ref_lib() is None:
        pytest.skip("reference harness not built")
    p = workloads.make_problem("disk_small")
    assert p["nt"] == 2000
    tr = _fwd(p)
    pr = oracle_prob(p, record="vz", damped_record=True)
    assert np.array_equal(tr, O.run_oracle(pr, fma_mode=1))
    ref = O.run_reference_labels(pr)
    assert rel_l2(tr, ref) < TOL
    # the sponge over the probe and both faces leaves no echo to pick
    t_lo, _, _ = workloads.bottom_echo_window(p)
    k = int(t_lo / p["dt"])
    assert np.abs(ref[k:]).max() < 1e-10 * np.abs(ref).max()


def test_disk_small_echo_variant_picks_identical_in_echo_window():
    from pefdtd import workloads
    if O.ref_lib() is None:
        pytest.skip("reference harness not built")
    p = workloads.make_problem(dict(workloads.WORKLOADS["disk_small"], sponge=6))
    tr = _fwd(p)
    tr64 = _fwd(p, dtype="float64")
    ref = O.run_reference_labels(oracle_prob(p, record="vz", damped_record=True))
    assert rel_l2(tr, ref) < TOL
    assert rel_l2(tr, tr64) < TOL
    (pa, pb, pc), t_lo, w_lo, w_hi = _echo_picks(p, tr, ref, tr64)
    k = int(t_lo / p["dt"])
    assert rel_l2(tr[k:], ref[k:]) < TOL          # the echo part alone
    for q in (pa, pb, pc):
        assert q[2] and w_lo <= q[0] <= w_hi      # a real maximum, inside the window
    assert pa[1] > 0.3 * np.abs(tr).max()          # a strong echo, not a tail
    assert round(pa[0] / p["dt"]) == round(pb[0] / p["dt"]) == round(pc[0] / p["dt"])
    assert abs(pa[0] - pb[0]) < PICK_REFINE_TOL * p["dt"]


def test_disk_prod_first_1800_steps_vs_reference_dense_fixture():
    from pefdtd import workloads
    if not os.path.exists(GOLD):
        pytest.skip("fixture not generated")
    g = np.load(GOLD)
    steps = int(g["steps"])
    p = workloads.make_problem("disk_prod", nt=steps)
    from golden.make_disk_prod_echo import input_digest
    assert input_digest(p, oracle_prob(p, record="vz", damped_record=True)) == str(g["digest"])
    tr = _fwd(p)
    tr64 = _fwd(p, dtype="float64")
    ref = g["trace"].reshape(-1, 1)
    assert rel_l2(tr, ref) < TOL
    assert rel_l2(tr, tr64) < TOL
    (pa, pb, pc), t_lo, w_lo, w_hi = _echo_picks(p, tr, ref, tr64)
    for q in (pa, pb, pc):
        assert q[2] and w_lo <= q[0] <= w_hi
    assert round(pa[0] / p["dt"]) == round(pb[0] / p["dt"]) == round(pc[0] / p["dt"])
    assert abs(pa[0] - pb[0]) < PICK_REFINE_TOL * p["dt"]


def _need_gpu_ref():
    if O.ref_gpu_lib() is None:
        pytest.skip("GPU reference harness not built")


def test_gpu_reference_harness_agrees_with_host_build():
    """The two builds of the reference's kernels differ only by FMA
    contraction."""
    from helpers import make_small
    _need_gpu_ref()
    if O.ref_lib() is None:
        pytest.skip("reference harness not built")
    p = make_small(nt=200, shape=(24, 30, 32), n_grains=9, sponge=4)
    for record in ("pressure", "vz"):
        pr = oracle_prob(p, record=record, damped_record=False)
        a, b = O.run_reference_labels_gpu(pr), O.run_reference_labels(pr)
        assert np.abs(b).max() > 0 and rel_l2(a, b) < 1e-5
        prd = oracle_prob(p, record=record, damped_record=True)
        a, b = O.run_reference_dense_gpu(prd), O.run_reference_dense(prd)
        assert rel_l2(a, b) < 1e-5


def test_disk_small_echo_variant_vs_gpu_reference():
    from pefdtd import workloads
    _need_gpu_ref()
    p = workloads.make_problem(dict(workloads.WORKLOADS["disk_small"], sponge=6))
    tr = _fwd(p)
    pr = oracle_prob(p, record="vz", damped_record=True)
    ref = O.run_reference_labels_gpu(pr)
    assert rel_l2(tr, ref) < TOL
    (pa, pb), t_lo, w_lo, w_hi = _echo_picks(p, tr, ref)
    assert pa[2] and pb[2] and w_lo <= pa[0] <= w_hi
    assert round(pa[0] / p["dt"]) == round(pb[0] / p["dt"])
    assert abs(pa[0] - pb[0]) < 1e-3 * p["dt"]


def test_disk_prod_full_length_vs_gpu_reference_dense():
    """disk_prod over its full 6000 steps against the reference's dense
    kernels on the GPU (500 grains: beyond the uint8 label path), the bottom
    echo picked identically, and the FP64 run of the same kernels."""
    from pefdtd import workloads
    _need_gpu_ref()
    p = workloads.make_problem("disk_prod")
    assert p["nt"] == 6000
    tr = _fwd(p)
    ref = O.run_reference_dense_gpu(oracle_prob(p, record="vz", damped_record=True))
    tr64 = _fwd(p, dtype="float64")
    assert rel_l2(tr, ref) < TOL
    assert rel_l2(tr, tr64) < TOL
    (pa, pb, pc), t_lo, w_lo, w_hi = _echo_picks(p, tr, ref, tr64)
    for q in (pa, pb, pc):
        assert q[2] and w_lo <= q[0] <= w_hi
    assert pa[1] > 0.3 * np.abs(tr).max()
    assert round(pa[0] / p["dt"]) == round(pb[0] / p["dt"]) == round(pc[0] / p["dt"])
    assert abs(pa[0] - pb[0]) < PICK_REFINE_TOL * p["dt"]
