"""Batched sweep on the GPU: every azimuth of a batch (records of different
lengths, 89-wide rows on the cp.async kernels) is bit-identical to its own
forward_fused_labels solve and to the oracle; the GPU labeller reproduces
the reference's exact labels (tests/golden/sweep_protocol.npz)."""
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CFG = dict(f0_mhz=0.5, ppw=6.0, az_start=0, az_stop=360, az_step=45, diameter_mm=80.0,
           thickness_mm=10.0, n_grains=12, sponge=10, seed=5)


def test_batched_sweep_matches_single_solves_and_oracle(tmp_path):
    from pefdtd import fdtd, specimen, sweep
    sweep.create("g", str(tmp_path), **CFG)
    cfg = sweep.load("g", str(tmp_path))
    assert sweep.run(cfg, batch=3, log=lambda *a: None) == "complete"
    assert len(sweep.done_azimuths(cfg)) == 8
    gold = np.load(os.path.join(GOLD, "sweep_protocol.npz"))
    f0 = cfg["f0_mhz"] * 1e6
    h = sweep.C_REF / f0 / cfg["ppw"]
    sp = specimen.DiskSpecimen(diameter_m=0.08, thickness_m=0.01, n_grains=12, size_cv=0.35,
                               concentration=3.93, spatial_corr=0.0, fabric_axis=(1, 0, 0), seed=5)
    build = sp.build(h, labeller="gpu")
    co = sweep.sweep_coeffs(cfg)
    for k, az in enumerate((45, 90)):
        s = sweep.azimuth_setup(cfg, build, co, az, labeller="gpu")
        lab = s["spec"]["mats"].astype(np.int32) - 1
        assert hashlib.sha256(lab.tobytes()).hexdigest() == str(gold[f"{az}_lab_sha"])
        spec = s["spec"]
        single = fdtd.forward_fused_labels(
            lab, s["axes"], s["h"], s["dt"], s["nt"],
            [(tuple(int(v) for v in np.unravel_index(i, lab.shape)), w)
             for i, w in zip(spec["src_idx"], spec["src_w"])],
            spec["wavelet"],
            [([tuple(int(v) for v in np.unravel_index(i, lab.shape)) for i in spec["rec_idx"]],
              spec["rec_w"])],
            coeffs=co, sponge_width=cfg["sponge"], damp_mask=spec["damp_volume"],
            mat_tables=(spec["Ct"], spec["rho_t"]))
        with np.load(os.path.join(tmp_path, "g", f"az{az:03d}.npz")) as z:
            assert np.array_equal(z["trace"], single[:, 0].astype(np.float32))
            assert float(z["dt"]) == s["dt"] and len(z["trace"]) == s["nt"]
            # figures from the device analysis against the host (reference) one
            E1, t1, coda, tail = sweep.analyse(np.asarray(z["trace"], float), s["dt"])
            assert float(z["t1_s"]) == t1 and abs(float(z["E1"]) - E1) <= 1e-11 * E1
            assert abs(float(z["coda_db"]) - coda) <= 1e-9
            assert (np.isnan(tail) and np.isnan(float(z["tail"]))) or abs(float(z["tail"]) - tail) <= 1e-11 * tail
        if k == 0:
            from oracle.oracle import problem_from_workload
            p = dict(lab=lab, mats=spec["mats"], Ct=spec["Ct"], rho_t=spec["rho_t"], h=s["h"],
                     dt=s["dt"], coeffs=co, sponge=cfg["sponge"], nt=s["nt"], record="pressure",
                     src_pts=[(tuple(int(v) for v in np.unravel_index(i, lab.shape)), w)
                              for i, w in zip(spec["src_idx"], spec["src_w"])],
                     rec_groups=[([tuple(int(v) for v in np.unravel_index(i, lab.shape))
                                   for i in spec["rec_idx"]], spec["rec_w"])],
                     wavelet=spec["wavelet"])
            ref = O.run_oracle(problem_from_workload(p, damped_record=False,
                                                     damp_mask=spec["damp_volume"]), fma_mode=1)
            assert np.array_equal(single, ref)
