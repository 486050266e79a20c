"""Generate tests/golden/fw_reference_2mhz.npz: the reference's own stored
full-wave traces of its ladder specimen with what a GPU test needs to
recompute them with this solver and apply the reference's acceptance gate.

The reference keeps four 2 MHz pressure traces of one specimen
(sim/ref/fw_fabric{00,25,50,100}.npz, written by
sim/fw_checks/fw_reference_2mhz.py:52-110): `ladder.standard_build()` (100 mm x
35 mm disk, 100 grains, seed 7, sim/model/ladder.py:68-72) at h = 3850 / 2e6 / 6,
`coda_convergence.build_grid` with a 10-cell sponge, the four fabric sets of
`ladder.standard_fabrics` (rng seed 11, :86-99), order 8, Ricker source,
fluid damping 0.02, a rim probe 6.35 mm across. Its gate
(sim/core/validate_labels.py:103-132): correlation > 0.999 and coda level
within 0.2 dB.

Stored here: the four traces with their dt, E1 and level, the four fabric
axis sets, and a digest of the solver grid built by this repository's
`specimen.DiskSpecimen(...).build(h, labeller="exact")` + `build_grid` (the
GPU labeller's argmin, which the test runs). The script also checks, against
the reference's own build (its CPU labeller): identical c-axes, this
repository's CPU-labeller restatement ("shortlist") identical cell for cell,
and how many cells the exact argmin assigns differently (the reference
documents a few, sim/core/specimen.py:303-310).

  PE_REFERENCE_ROOT=<reference checkout> python tests/golden/make_fw_reference.py
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "fw_reference_2mhz.npz")
TAGS = ("00", "25", "50", "100")
SPEC = dict(diameter_m=0.100, thickness_m=0.035, n_grains=100, size_cv=0.35, concentration=3.93,
            spatial_corr=0.0, fabric_axis=(1, 0, 0), seed=7)
H = 3850.0 / 2e6 / 6.0
SPONGE = 10


def grid_digest(lab):
    return hashlib.sha256(np.ascontiguousarray(lab, np.int32).tobytes()).hexdigest()


def main():
    ref = os.environ.get("PE_REFERENCE_ROOT")
    if not ref or not os.path.isdir(os.path.join(ref, "sim", "ref")):
        raise SystemExit("set PE_REFERENCE_ROOT to the reference checkout (it reads sim/ref and imports sim/model)")
    sys.path[:0] = [os.path.join(ref, "sim", d) for d in ("core", "model", "pipeline", "fw_checks")]
    sys.path[:0] = [os.path.join(ref, "vendor"), ROOT, os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200")]
    import ladder                      # the reference's
    from pefdtd import specimen        # this repository's

    t0 = time.time()
    rb = ladder.standard_build()       # reference DiskSpecimen, its CPU labeller
    print(f"reference build {rb['labels'].shape}: {time.time() - t0:.0f} s", flush=True)
    t0 = time.time()
    sp = specimen.DiskSpecimen(**SPEC)
    ours_sl = sp.build(H, labeller="shortlist")
    ours = sp.build(H, labeller="exact")
    print(f"own builds: {time.time() - t0:.0f} s", flush=True)
    assert np.array_equal(ours["axes"], rb["axes"]), "c-axes differ from the reference build"
    assert np.array_equal(ours_sl["labels"], rb["labels"]), "CPU labeller restatement differs"
    n_diff = int((ours["labels"] != rb["labels"]).sum())
    print(f"exact argmin vs the reference's CPU labeller: {n_diff} of {rb['labels'].size} cells", flush=True)
    lab, nd, m = specimen.build_grid(ours["labels"], H, H, SPONGE)
    fabrics = np.stack(ladder.standard_fabrics(rb["axes"]))
    traces, dts, e1, lvl, frac = [], [], [], [], []
    for tag in TAGS:
        d = np.load(os.path.join(ref, "sim", "ref", f"fw_fabric{tag}.npz"))
        assert float(d["fluid_damp"]) == 0.02 and int(d["order"]) == 8 and int(d["seed_specimen"]) == 7
        traces.append(np.asarray(d["trace"], np.float64).ravel())
        dts.append(float(d["dt"]))
        e1.append(float(d["E1"]))
        lvl.append(float(d["level_db"]))
        frac.append(float(d["frac"]))
    assert len({len(t) for t in traces}) == 1 and len(set(dts)) == 1
    np.savez_compressed(OUT, traces=np.stack(traces), dt=dts[0], E1=np.array(e1), level_db=np.array(lvl),
                        frac=np.array(frac), axes=fabrics, h=H, sponge=SPONGE, fluid_damp=0.02, f0=2e6,
                        grid_shape=np.array(lab.shape), nd=nd, m=m, grid_digest=grid_digest(lab),
                        labeller_cells_differing=n_diff)
    print(f"wrote {OUT}: grid {lab.shape}, {len(traces[0])} samples, dt {dts[0]:.6e}", flush=True)


if __name__ == "__main__":
    main()
