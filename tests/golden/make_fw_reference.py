"""Generate tests/golden/fw_reference.npz: the reference's own stored
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

The six azimuth traces sim/ref/fw_az{17,31,47,62,76,90}.npz
(sim/pipeline/azimuth_sweep.py:62-120: the same specimen resampled by
`rotation_test.rotated_grid`, dt from `safe_dt_labels` per azimuth) are
stored too, with the digests of the rotated grids and the c-axes in both
rotation conventions: `axes @ R` (the reference's current `rotated_grid`,
sim/core/rotation_test.py:66-75, 132-134) and `axes @ R.T`, the convention
that code replaced, which the stored azimuth traces were computed with (they
are dated before the fix, azimuth_sweep.py:18).

Two traces of the same specimen at the probe's higher frequencies are stored
as well: sim/ref/fw_3mhz.npz (sim/fw_checks/freq_blips.py:170-207, 46 M
cells, 5937 steps) and sim/ref/fw_5mhz_fabric00.npz
(sim/fw_checks/fw_reference_5mhz.py:33-80, 194 M cells, 9895 steps), each
with the digest and c-axes of this repository's build at its spacing, and
the 5 MHz run cropped to the E1 corridor |y| <= 27 mm about the beam axis
(sim/ref/fw_5mhz_e1corridor.npz, sim/fw_checks/fw_e1_corridor_validate.py:
49-104).

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
OUT = os.path.join(HERE, "fw_reference.npz")
TAGS = ("00", "25", "50", "100")
AZIMUTHS = (17, 31, 47, 62, 76, 90)
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
    from rotation_test import rotated_grid as ref_rotated_grid   # the reference's
    az_rot, az_tr, az_dt, az_lvl, az_dig, az_cur, az_leg = [], [], [], [], [], [], []
    for rot in AZIMUTHS:
        d = np.load(os.path.join(ref, "sim", "ref", f"fw_az{rot:02d}.npz"))
        assert float(d["fluid_damp"]) == 0.02 and int(d["rot_deg"]) == rot
        rl, rnd, rm, rax = ref_rotated_grid(dict(labels=ours["labels"], axes=ours["axes"], h=H), H, SPONGE, rot)
        ol, ond, om, oax = specimen.rotated_grid(ours["labels"], ours["axes"], H, H, SPONGE, rot)
        assert np.array_equal(rl, ol) and np.array_equal(rax, oax) and (rnd, rm) == (ond, om)
        a = np.radians(rot)
        R = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
        az_rot.append(rot)
        az_tr.append(np.asarray(d["trace"], np.float64).ravel())
        az_dt.append(float(d["dt"]))
        az_lvl.append(float(d["level_db"]))
        az_dig.append(grid_digest(ol))
        az_cur.append(oax)
        az_leg.append(ours["axes"] @ R.T)
    az_len = np.array([len(t) for t in az_tr])      # nt differs with dt per azimuth
    az_pad = np.zeros((len(az_tr), int(az_len.max())))
    for i, t in enumerate(az_tr):
        az_pad[i, :len(t)] = t
    hf = {}
    for tag, f0 in (("fw_3mhz", 3e6), ("fw_5mhz_fabric00", 5e6)):
        d = np.load(os.path.join(ref, "sim", "ref", f"{tag}.npz"))
        hh = float(d["h"])
        assert abs(hh - 3850.0 / f0 / 6.0) < 1e-15 and int(d["order"]) == 8 and int(d["seed_specimen"]) == 7
        t0 = time.time()
        bh = sp.build(hh, labeller="exact")
        gl, _, _ = specimen.build_grid(bh["labels"], hh, hh, SPONGE)
        print(f"{tag}: grid {gl.shape}, {time.time() - t0:.0f} s", flush=True)
        key = "f3" if f0 == 3e6 else "f5"
        hf[f"{key}_trace"] = np.asarray(d["trace"], np.float64).ravel()
        hf[f"{key}_dt"] = float(d["dt"])
        hf[f"{key}_h"] = hh
        hf[f"{key}_f0"] = f0
        hf[f"{key}_axes"] = bh["axes"]
        hf[f"{key}_grid_digest"] = grid_digest(gl)
        del bh, gl
    d = np.load(os.path.join(ref, "sim", "ref", "fw_5mhz_e1corridor.npz"))
    assert abs(float(d["dt"]) - hf["f5_dt"]) < 1e-20
    hf["f5c_trace"] = np.asarray(d["trace"], np.float64).ravel()
    hf["f5c_half_w"] = float(d["half_w"])
    np.savez_compressed(OUT, **hf, traces=np.stack(traces), dt=dts[0], E1=np.array(e1), level_db=np.array(lvl),
                        frac=np.array(frac), axes=fabrics, h=H, sponge=SPONGE, fluid_damp=0.02, f0=2e6,
                        grid_shape=np.array(lab.shape), nd=nd, m=m, grid_digest=grid_digest(lab),
                        labeller_cells_differing=n_diff, az_rot=np.array(az_rot), az_traces=az_pad, az_len=az_len,
                        az_dt=np.array(az_dt), az_level_db=np.array(az_lvl), az_grid_digest=np.array(az_dig),
                        az_axes_current=np.stack(az_cur), az_axes_legacy=np.stack(az_leg))
    print(f"wrote {OUT}: grid {lab.shape}, {len(traces[0])} samples, dt {dts[0]:.6e}", flush=True)


if __name__ == "__main__":
    main()
