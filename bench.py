#!/usr/bin/env python
"""Throughput of the label-indexed anisotropic elastic FDTD step on B200.

Metric: Gcell-updates/s = cells x steps / device time (every cell of the grid
counts, fluid and sponge included, as the reference counts them). One bench
"step" is one time step of the solver over the whole workload grid.

Default workload: disk_prod (160 x 256 x 256 cells, 500 grains, girdle
fabric; see pefdtd/workloads.py), the configuration the single-solve
throughput is quoted on. Its nine FP32 state fields are 377 MB, three times
the 126 MB L2, so every step streams from HBM and no L2 flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank advances its own
independent solve of the workload: a single solve does not shard, batches of
solves do (scaling "weak"); the value is all ranks' cell updates over the
slowest rank's device time.

--impl reference runs the reference's own update kernels, compiled for the
host CPU from the reference sources (oracle/_ref; oracle port if absent), on
all host cores, rank 0 only, time-boxed.

--sweep N prints one line comparing an N-solve sweep of the workload grid
run batched (one launch pair per step for all solves, pefdtd.batch) against
the plain loop (one solve at a time, each created, run and read back in
turn); both timings include solver set-up and trace download. --uneven adds
24 solves of uneven grids (128 x 128 x 96 ... 256 x 256 x 160, 100-800
grains, Watson kappa 0-20) to the batch.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

ALG_BYTES_STEP = 74      # 9 f32 fields read + written, u16 label read, per cell-update
ALG_BYTES_STRESS = 62    # v read 12, s read 24 + write 24, label 2
ALG_BYTES_VEL = 50       # s read 24, v read 12 + write 12, label 2
SPLIT_FROM = 300         # the per-kernel split is taken from this step on (filled wavefield)
SWEEP_STEPS = 200        # steps per solve of the compact 36-azimuth sweep in the default line


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # PE_CLOCKS_DIR keeps the raw samples (e.g. to attach them to a run);
        # by default they go to the system temporary directory
        self.path = os.path.join(os.environ.get("PE_CLOCKS_DIR") or tempfile.gettempdir(),
                                 f"pefdtd_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def _problem(workload, nt, use_gpu=None):
    from pefdtd import workloads
    return workloads.make_problem(workload, nt=nt, use_gpu=use_gpu)


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.lower().startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    import platform
    return platform.processor() or "unknown"


def _device_solve(p, nt_total):
    from pefdtd.fdtd import DeviceSolve, _flat_probe
    from pefdtd.damping import sponge_axis_profiles
    shape = p["lab"].shape
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], np.float32)
    solve = DeviceSolve(p["mats"], p["Ct"], p["rho_t"], p["h"], p["dt"], p["coeffs"], s_idx, s_w,
                        r_off, r_idx, r_w, record=p["record"], damped_record=True,
                        sponge=sponge_axis_profiles(shape, p["sponge"]))
    solve.set_wavelet(p["wavelet"][:nt_total])
    return solve


def _fp64_check(p, nt):
    """The workload at its full length, FP32 against an FP64 run of the same
    kernels on the same inputs: relative L2 of the traces, and the
    Hilbert-envelope pick of the disk's bottom-face echo in both (searched
    past the transmitted burst, required inside the echo window)."""
    from pefdtd import wavelets, workloads
    from pefdtd.damping import sponge_axis_profiles
    from pefdtd.fdtd import DeviceSolve, _flat_probe
    shape = p["lab"].shape
    spec = p["spec"]
    wav = wavelets.hann_tone_burst(nt, p["dt"], spec["f0"], n_cycles=spec["n_cycles"])
    out = {}
    for dtype, npdt in (("float32", np.float32), ("float64", np.float64)):
        s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], npdt)
        sv = DeviceSolve(p["mats"], p["Ct"], p["rho_t"], p["h"], p["dt"], p["coeffs"], s_idx, s_w, r_off,
                         r_idx, r_w, record=p["record"], damped_record=True,
                         sponge=sponge_axis_profiles(shape, p["sponge"]), dtype=dtype)
        try:
            sv.set_wavelet(wav)
            sv.run(0, nt)
            sv.check_status()
            out[dtype] = np.asarray(sv.traces_numpy(nt), float)[:, 0]
        finally:
            sv.close()
    a, b = out["float32"], out["float64"]
    rel = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    t = np.arange(nt) * p["dt"]
    t_lo, w_lo, w_hi = workloads.bottom_echo_window(p)
    pa = wavelets.pick_peak(t, a, t_lo=t_lo, dt=p["dt"])
    pb = wavelets.pick_peak(t, b, t_lo=t_lo, dt=p["dt"])
    k_lo, k_hi = int(t_lo / p["dt"]), nt
    same = bool(pa[2] == pb[2] and round(pa[0] / p["dt"]) == round(pb[0] / p["dt"]))
    in_win = bool(w_lo <= pa[0] <= w_hi and w_lo <= pb[0] <= w_hi)
    echo_rel = float(np.linalg.norm(a[k_lo:k_hi] - b[k_lo:k_hi]) / max(np.linalg.norm(b[k_lo:k_hi]), 1e-300))
    return {"steps": nt, "trace_rel_l2": rel, "echo_window_s": [w_lo, w_hi], "pick_search_from_s": t_lo,
            "echo_pick_s_f32_f64": [pa[0], pb[0]], "echo_pick_identical": same,
            "echo_pick_in_window": in_win, "echo_rel_l2_after_burst": echo_rel,
            "echo_to_burst_envelope": float(pb[1] / max(np.abs(b).max(), 1e-300))}


def _e2e(p, steps, warm=True):
    """Same metric through the public C ABI host entry (pe_forward_host):
    pinned host labels/tables/probe in, traces out, all inside the timing
    (device allocation, uploads, graph capture, the steps, download, frees).
    One untimed 3-step call first, so that one-time process initialisation
    (kernel attributes, driver entry points) is not charged to the run."""
    if warm:
        _e2e(p, 3, warm=False)
    import torch
    from pefdtd import _capi
    from pefdtd.damping import sponge_axis_profiles
    from pefdtd.fdtd import _flat_probe
    L = _capi.lib()
    shape = p["lab"].shape
    nz, ny, nx = shape
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], np.float32)
    lab_pin = torch.from_numpy(p["mats"].astype(np.uint16).view(np.int16)).pin_memory()
    tr_pin = torch.zeros((steps, len(r_off) - 1), dtype=torch.float32).pin_memory()
    Ct = np.ascontiguousarray(p["Ct"], np.float32)
    rho = np.ascontiguousarray(p["rho_t"], np.float32)
    sp = [np.ascontiguousarray(a, np.float32) for a in sponge_axis_profiles(shape, p["sponge"])]
    wav = np.ascontiguousarray(p["wavelet"][:steps], np.float32)
    cfg = _capi.PeConfig()
    cfg.nz, cfg.ny, cfg.nx = shape
    cfg.dtype = _capi.PE_F32
    cfg.n_coeffs = len(p["coeffs"])
    for j, c in enumerate(p["coeffs"]):
        cfg.coeffs[j] = float(c)
    cfg.h, cfg.dt = p["h"], p["dt"]
    cfg.record = _capi.REC_KIND[p["record"]]
    cfg.damped_record = 1
    cfg.n_mat = len(rho)
    md = _capi.PeMedium()
    md.ctab, md.rho = _capi.ptr(Ct), _capi.ptr(rho)
    md.sponge_z, md.sponge_y, md.sponge_x = [_capi.ptr(a) for a in sp]
    pr = _capi.PeProbe()
    pr.n_src, pr.src_idx, pr.src_w = len(s_idx), _capi.ptr(s_idx), _capi.ptr(s_w)
    pr.n_groups, pr.rec_off, pr.rec_idx, pr.rec_w = len(r_off) - 1, _capi.ptr(r_off), _capi.ptr(r_idx), _capi.ptr(r_w)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = L.pe_forward_host(_capi.C.byref(cfg), lab_pin.data_ptr(), None, _capi.C.byref(md),
                           _capi.C.byref(pr), _capi.ptr(wav), steps, tr_pin.data_ptr())
    el = time.perf_counter() - t0
    _capi.check(rc)
    ncell = nz * ny * nx
    h2d = ncell * 2 + Ct.nbytes + rho.nbytes + sum(a.nbytes for a in sp) + wav.nbytes \
        + s_idx.nbytes + s_w.nbytes + r_off.nbytes + r_idx.nbytes + r_w.nbytes
    return {"value": ncell * steps / el / 1e9, "unit": "Gcell-updates/s",
            "h2d_bytes_per_step": int(h2d // steps), "d2h_bytes_per_step": int(tr_pin.nbytes // steps),
            "steps": steps, "wall_s": el, "api": "pe_forward_host (C ABI, host buffers)"}


def _cpu_run(p, budget_s, max_steps, warmup=3):
    """Reference kernels on the host (oracle/_ref), else the C oracle port;
    `warmup` untimed steps (which also size the sample), then a time-boxed
    timed run. Returns (Gcell/s, steps, cores, kind, sample)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    ncell = int(np.prod(p["lab"].shape))
    kind = "reference" if O.ref_lib() is not None else "port"
    dense = p["mats"].max() > 255

    def run(nsteps):
        q = dict(p)
        q["nt"] = nsteps
        q["wavelet"] = p["wavelet"][:nsteps]
        pr = O.problem_from_workload(q, record=p["record"], damped_record=True)
        t0 = time.perf_counter()
        if kind == "reference":
            (O.run_reference_dense if dense else O.run_reference_labels)(pr, n_threads=cores)
        else:
            O.run_oracle(pr, n_threads=cores)
        return time.perf_counter() - t0

    w = max(1, int(warmup))
    t1 = run(w) / w                     # warm-up steps, which also size the sample
    n = int(max(2, min(max_steps, len(p["wavelet"]), budget_s / max(t1, 1e-3))))
    el = run(n)
    which = ("the reference's dense update kernels (strains, stress_acc, vel_update)"
             if dense else "the reference's label-path kernels (strains_zp, stress_lab_u, vel_zp)")
    sample = (f"{n} time steps of the full {p['name']} grid ({ncell} cells), FP32, {which} "
              f"compiled for the host with gcc -O2 -fopenmp, {cores} threads"
              if kind == "reference" else
              f"{n} time steps of the full {p['name']} grid, C oracle port, {cores} threads")
    return ncell * n / el / 1e9, n, cores, kind, sample


def _uneven_specs(n=24):
    """Uneven disks: grids from 128 x 128 x 96 to 256 x 256 x 160 (rows of
    16-byte multiples), 100-800 grains, Watson kappa 0-20, seeded."""
    out = []
    for i in range(n):
        f = i / max(1, n - 1)
        nxy = int(round((128 + 128 * f) / 16)) * 16
        nz = int(round((96 + 64 * f) / 8)) * 8
        h = 0.1e-3
        d = (nxy - 70) * h
        out.append(dict(shape=(nz, nxy, nxy), h=h, diameter=d, height=min(10e-3, (nz - 70) * h),
                        n_grains=int(100 + 700 * ((i * 7) % n) / max(1, n - 1)),
                        fabric=("watson", 30.0, 20.0 * ((i * 5) % n) / max(1, n - 1)),
                        f0=2.25e6, n_cycles=5, nt=6000, sponge=32, aperture=6e-3, seed=100 + i))
    return out


def _sweep(args):
    """Batched vs plain N-solve sweep (one line of JSON)."""
    import torch
    from pefdtd import batch, workloads
    from pefdtd.fdtd import _flat_probe
    from pefdtd.damping import sponge_axis_profiles
    K = int(args.steps)
    base = workloads.make_problem(args.workload, nt=K + 8)
    probs = [base] * int(args.sweep)
    if args.uneven:
        probs = probs + [workloads.make_problem(sp, nt=K + 8) for sp in _uneven_specs()]
    cells = sum(int(np.prod(p["lab"].shape)) for p in probs)
    specs = [batch.spec_from_problem(p) for p in probs]

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = []
    for p in probs:
        shape = p["lab"].shape
        s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], np.float32)
        from pefdtd.fdtd import DeviceSolve
        sv = DeviceSolve(p["mats"], p["Ct"], p["rho_t"], p["h"], p["dt"], p["coeffs"], s_idx, s_w,
                         r_off, r_idx, r_w, record=p["record"], damped_record=True,
                         sponge=sponge_axis_profiles(shape, p["sponge"]))
        sv.set_wavelet(p["wavelet"][:K])
        sv.run(0, K)
        plain.append(sv.traces_numpy(K))
        sv.close()
        del sv
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0

    # warm-up of the batch paths (kernel attributes, graph capture) on two solves
    wb = batch.BatchSolver(specs[:2])
    try:
        wb.set_persistent(True)
        wb.run(0, 4)
        wb.traces_numpy(4)
    finally:
        wb.close()
    t_modes, gots = {}, {}
    for persistent in (False, True):
        t0 = time.perf_counter()
        b = batch.BatchSolver(specs)
        try:
            b.set_persistent(persistent)
            b.run(0, K)
            gots[persistent] = b.traces_numpy(K)
        finally:
            b.close()
        torch.cuda.synchronize()
        t_modes[persistent] = time.perf_counter() - t0
    t_batch, got = min(t_modes.values()), gots[True]
    same = all(np.array_equal(a, g[:K]) and np.array_equal(g, q) for a, g, q in zip(plain, got, gots[False]))
    return {"metric": "sweep Gcell-updates/s, batched vs plain loop", "unit": "Gcell-updates/s",
            "solves": len(probs), "steps": K, "cells_per_step": cells,
            "plain": cells * K / t_plain / 1e9, "batched": cells * K / t_batch / 1e9,
            "speedup": t_plain / t_batch, "plain_s": t_plain, "batched_s": t_batch,
            "batched_per_step_s": t_modes[False], "batched_persistent_s": t_modes[True],
            "traces_identical": bool(same),
            "config": {"workload": args.workload, "uneven24": bool(args.uneven),
                       "timing": "wall clock, set-up and trace download included, synchronised"}}


def _azimuth_host(base, az):
    """The reference's per-azimuth set-up on the host (sweep_runner.py:322-390):
    the label volume and the c-axes turned by -az (NumPy resample), the
    material tables, the probe on the rotated grid."""
    from pefdtd import inversion, materials, workloads
    lab = inversion.rotate_labels(base["lab"], az)
    a = np.radians(az)
    R = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
    axes = np.asarray(base["axes"], float) @ R
    Ct, rho = materials.material_tables(axes)
    pts = workloads.top_probe(lab, base["h"], base["spec"]["aperture"])
    w = 1.0 / len(pts)
    return dict(base, lab=lab, mats=(lab + 1).astype(np.uint16), axes=axes, Ct=Ct, rho_t=rho,
                src_pts=[(q, w) for q in pts], rec_groups=[(pts, np.full(len(pts), w))])


def _azimuth_specs_device(base, azs):
    """The batched set-up: one upload of the label volume, every azimuth's
    rotated labels gathered on the device (the same nearest-cell resample),
    tables and probe (one plane) on the host."""
    import torch
    from pefdtd import batch, inversion, materials, workloads
    nz, ny, nx = base["lab"].shape
    lab_d = torch.from_numpy(np.ascontiguousarray(base["lab"], np.int32)).cuda()
    iz = int(np.nonzero((base["lab"] >= 0).any(axis=(1, 2)))[0][0])
    X, Y = np.meshgrid(np.arange(nx) - (nx - 1) / 2.0, np.arange(ny) - (ny - 1) / 2.0, indexing="xy")
    specs = []
    for az in azs:
        a = np.radians(az)
        ca, sa = np.cos(a), np.sin(a)
        xs = np.rint(ca * X - sa * Y + (nx - 1) / 2.0).astype(np.int64)
        ys = np.rint(sa * X + ca * Y + (ny - 1) / 2.0).astype(np.int64)
        ok = (xs >= 0) & (xs < nx) & (ys >= 0) & (ys < ny)
        flat = torch.from_numpy(np.where(ok, np.clip(ys, 0, ny - 1) * nx + np.clip(xs, 0, nx - 1), -1)).cuda()
        src = lab_d.reshape(nz, ny * nx)[:, flat.clamp(min=0).reshape(-1)].reshape(nz, ny, nx)
        mats = torch.where(flat.reshape(1, ny, nx) >= 0, src + 1, torch.zeros_like(src))
        plane = inversion.rotate_labels(base["lab"][iz:iz + 1], az)
        full = np.full((iz + 1, ny, nx), -1, np.int32)
        full[iz] = plane[0]
        pts = workloads.top_probe(full, base["h"], base["spec"]["aperture"])
        w = 1.0 / len(pts)
        R = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])
        Ct, rho = materials.material_tables(np.asarray(base["axes"], float) @ R)
        p = dict(base, Ct=Ct, rho_t=rho, src_pts=[(q, w) for q in pts],
                 rec_groups=[(pts, np.full(len(pts), w))])
        sp = batch.spec_from_problem(p)
        sp["mats"] = mats
        specs.append(sp)
    return specs


def _sweep_compact(K, workload="disk_small", n_az=36):
    """A 36-azimuth sweep of one disk and its misfit gradients, each run as
    the reference runs it (one azimuth at a time: host set-up, upload, solve,
    read back) and batched (device-side set-up, one batch). Wall clock,
    synchronised; traces and gradients compared between the arms."""
    import torch
    from pefdtd import adjoint, batch, inversion, workloads
    base = workloads.make_problem(workload, nt=K)
    azs = [360.0 * i / n_az for i in range(n_az)]
    cells = int(np.prod(base["lab"].shape))
    # warm-up of both paths (library, allocator, graph capture)
    sv = _device_solve(_azimuth_host(base, 0.0), K)
    sv.run(0, 8)
    sv.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = []
    for az in azs:
        sv = _device_solve(_azimuth_host(base, az), K)
        sv.run(0, K)
        plain.append(sv.traces_numpy(K))
        sv.close()
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    def batched(persistent):
        t0 = time.perf_counter()
        b = batch.BatchSolver(_azimuth_specs_device(base, azs))
        try:
            b.set_persistent(persistent)
            b.run(0, K)
            got = b.traces_numpy(K)
        finally:
            b.close()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, got

    batched(True)   # warm-up of the batch paths
    t_step, got_step = batched(False)
    t_batch, got = batched(True)
    same = all(np.array_equal(a, g[:K]) and np.array_equal(g, q) for a, g, q in zip(plain, got, got_step))
    out = {"azimuths": n_az, "steps": K, "workload": workload, "cells_per_solve": cells,
           "plain_s": t_plain, "batched_s": t_batch, "speedup": t_plain / t_batch,
           "batched_per_step_launches_s": t_step, "traces_identical": bool(same),
           "plain": "per azimuth: host rotation of labels and axes, tables, probe, upload, solve, read back",
           "batched": "labels uploaded once and rotated on the device, one batch of all azimuths, "
                      "one persistent launch per graph chunk (per-step launches timed beside it)"}
    # the gradients of the same sweep (misfit against the traces of a
    # perturbed fabric), one at a time and batched
    disk = inversion.Disk(workload, azs, nt=K, dtype="float32", checkpoint_every=200)
    th, ph = adjoint.angles_from_axes(disk.true_axes)
    th_t, ph_t = torch.as_tensor(th), torch.as_tensor(ph)
    c21s = [inversion.tables21(th_t, ph_t, az).numpy() for az in azs]
    dobs = [g[:K] * 1.01 for g in got]
    adjoint.misfit_gradients(disk.problems[:1], c21s[:1], dobs[:1])   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    one = [adjoint.misfit_gradients([p], [c], [d])[0] for p, c, d in zip(disk.problems, c21s, dobs)]
    torch.cuda.synchronize()
    tg_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    many = adjoint.misfit_gradients(disk.problems, c21s, dobs)
    torch.cuda.synchronize()
    tg_batch = time.perf_counter() - t0
    dev = max(float(np.abs(g - q).max() / max(np.abs(q).max(), 1e-300)) for (_, g), (_, q) in zip(many, one))
    out["gradients"] = {"solves": n_az, "steps": K, "plain_s": tg_plain, "batched_s": tg_batch,
                        "speedup": tg_plain / tg_batch, "max_rel_grad_diff": dev,
                        "checkpoint_every": 200}
    out["sweep_plus_gradients_speedup"] = (t_plain + tg_plain) / (t_batch + tg_batch)
    return out


def _traces(args):
    """Device vs host post-processing of N records of the workload's length
    (sweep analysis and high-passed picks; one line of JSON)."""
    import torch
    from pefdtd import traces, wavelets
    n, N, dt = 6000, int(args.traces), 1.0e-8
    rng = np.random.default_rng(7)
    t = np.arange(n) * dt
    host = []
    for i in range(N):
        x = 0.2 + 0.01 * rng.standard_normal(n)
        tau = t - (51.9e-6 + 0.3e-6 * rng.standard_normal())
        m = (tau >= 0) & (tau <= 2.2e-6)
        x[m] += 0.5 * (1 - np.cos(2 * np.pi * tau[m] / 2.2e-6)) * np.sin(2 * np.pi * 2.25e6 * tau[m])
        host.append(x.astype(np.float32))
    dev = [torch.from_numpy(x).cuda() for x in host]

    def device_pass():
        a = traces.analyse(dev, dt)
        p = traces.pick_peaks(t, dev, t_lo=30e-6, f_lo=0.3e6)
        return a, p

    for _ in range(3):
        device_pass()
    torch.cuda.synchronize()
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        a_dev, p_dev = device_pass()
    torch.cuda.synchronize()
    t_dev = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    a_host = [wavelets.analyse_trace(np.asarray(x, float), dt) for x in host]
    p_host = [wavelets.pick_peak(t, x, t_lo=30e-6, dt=dt, f_lo=0.3e6) for x in host]
    t_host = time.perf_counter() - t0
    same_t1 = all(a[1] == b[1] for a, b in zip(a_dev, a_host))
    same_pick = all(abs(a[0] - b[0]) <= 1e-6 * dt and a[2] == b[2] for a, b in zip(p_dev, p_host))
    return {"metric": "traces post-processed/s (analysis + high-passed pick)", "unit": "traces/s",
            "traces": N, "samples": n, "device": N / t_dev, "host": N / t_host,
            "speedup": t_host / t_dev, "device_ms": t_dev * 1e3, "host_ms": t_host * 1e3,
            "host_cores": 1, "arrivals_identical": bool(same_t1), "picks_identical": bool(same_pick),
            "config": {"timing": "wall clock; device: f32 records resident on the GPU, results read back; "
                                 "host: the reference's SciPy computations, one thread"}}


def _gradients(args):
    """Misfit gradients of an N-azimuth sweep of one disk (the gradient
    configuration: checkpoints every 200 steps, recomputation, the memory
    plan of pefdtd.adjoint deciding waves, two-level checkpoints and host
    offload for the free HBM): one at a time vs batched (one line of JSON)."""
    import torch
    from pefdtd import adjoint, inversion
    K = int(args.steps)
    n = int(args.gradients)
    azs = [360.0 * i / n for i in range(n)]
    disk = inversion.Disk(args.workload, azs, nt=K, dtype="float32", checkpoint_every=200)
    th, ph = adjoint.angles_from_axes(disk.true_axes)
    th_t, ph_t = torch.as_tensor(th), torch.as_tensor(ph)
    c21s = [inversion.tables21(th_t, ph_t, az).numpy() for az in azs]
    # observed data: the traces of the same disk with its c-axes re-drawn
    rng = np.random.default_rng(int(disk.base["spec"]["seed"]) + 1)
    th2, ph2 = inversion.isotropic_angles(disk.n_grains, rng)
    dobs = [pr.traces_numpy(inversion.tables21(torch.as_tensor(th2), torch.as_tensor(ph2), az).numpy())
            for pr, az in zip(disk.problems[:1], azs[:1])] * n
    free = torch.cuda.mem_get_info()[0]
    budget = int(0.8 * free)
    waves = adjoint.plan_waves(disk.problems, budget)
    adjoint.misfit_gradients(disk.problems[:1], c21s[:1], dobs[:1])   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    many = adjoint.misfit_gradients(disk.problems, c21s, dobs, memory_budget=budget)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    peak = torch.cuda.max_memory_allocated()
    n_plain = min(n, int(args.plain_solves) if args.plain_solves else n)
    t0 = time.perf_counter()
    one = [adjoint.misfit_gradients([p], [c], [d], memory_budget=budget)[0]
           for p, c, d in zip(disk.problems[:n_plain], c21s[:n_plain], dobs[:n_plain])]
    torch.cuda.synchronize()
    t_plain = (time.perf_counter() - t0) * n / n_plain
    dev = max(float(np.abs(g - q).max() / max(np.abs(q).max(), 1e-300)) for (_, g), (_, q) in zip(many, one))
    # chained to every grain's (theta, phi) and to the 3 fabric parameters
    # (tilt, azimuth, log concentration about the grains' own axes)
    t0 = time.perf_counter()
    th_l = torch.tensor(th, requires_grad=True)
    ph_l = torch.tensor(ph, requires_grad=True)
    fab = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    base = torch.as_tensor(inversion.axes_of(th, ph))
    th_f, ph_f = adjoint.theta_phi_torch(adjoint.fabric_axes(fab, base))
    loss = 0.0
    for az, (_, G) in zip(azs, many):
        Gt = torch.as_tensor(np.asarray(G))
        loss = loss + (inversion.tables21(th_l, ph_l, az) * Gt[:disk.n_grains + 1]).sum()
        loss = loss + (inversion.tables21(th_f, ph_f, az) * Gt[:disk.n_grains + 1]).sum()
    loss.backward()
    t_chain = time.perf_counter() - t0
    shape = disk.base["lab"].shape
    plan = sorted({opt for w in waves for _, opt in w})
    return {"metric": "misfit + gradient solves/s, batched vs plain loop", "unit": "solves/s",
            "solves": n, "steps": K, "grid": list(shape), "grains": disk.n_grains,
            "angles": 2 * disk.n_grains, "plain": n / t_plain, "batched": n / t_batch,
            "speedup": t_plain / t_batch, "plain_s": t_plain, "batched_s": t_batch,
            "plain_solves_timed": n_plain, "max_rel_grad_diff": dev,
            "angle_gradient": {"n": int(2 * disk.n_grains), "norm": float(torch.cat([th_l.grad, ph_l.grad]).norm()),
                               "fabric_params": [float(v) for v in fab.grad], "chain_s": t_chain},
            "waves": [len(w) for w in waves], "plan_inner_offload": [list(o) for o in plan],
            "bytes_per_solve_unplanned": adjoint.adjoint_bytes(shape, K, 200),
            "device_budget_bytes": budget, "peak_allocated_bytes": int(peak),
            "config": {"workload": args.workload, "dtype": "f32", "checkpoint_every": 200,
                       "timing": "wall clock; solver creation, forward, adjoint and gradient download included"}}


def _inversion_specs(n):
    """Disks of mixed sizes and fabrics for the inversion (seeded): grids from
    64 x 96 x 96 to 80 x 128 x 128 at h = 0.2 mm, 40-120 grains,
    single-maximum (Watson kappa 5-20 about an axis 30 deg from z) and girdle
    fabrics, 1 MHz 3-cycle burst, 8-cell sponge (both disk faces outside it,
    so the bottom echo reaches the probe)."""
    out = []
    for i in range(n):
        f = i / max(1, n - 1)
        nxy = int(round((96 + 32 * f) / 16)) * 16
        nz = int(round((64 + 16 * f) / 8)) * 8
        h = 0.2e-3
        fabric = ("watson", 30.0, 5.0 + 15.0 * f) if i % 2 == 0 else ("girdle", 20.0, 10.0)
        out.append(dict(shape=(nz, nxy, nxy), h=h, diameter=(nxy - 22) * h, height=(nz - 22) * h,
                        n_grains=int(40 + 80 * ((3 * i) % n) / max(1, n - 1)), fabric=fabric,
                        f0=1.0e6, n_cycles=3, nt=2000, sponge=8, aperture=6e-3, seed=300 + i))
    return out


def _inversion(args):
    """The batched gradient fabric inversion (pefdtd.inversion): D disks x A
    azimuths, L-BFGS on every grain's (theta, phi) from an isotropic fabric,
    batched; the plain loop's evaluation timed once beside it (one line)."""
    import torch
    from pefdtd import inversion
    D, A, K, I = int(args.inversion), int(args.azimuths), int(args.steps), int(args.iterations)
    azs = [360.0 * i / A for i in range(A)]
    disks = [inversion.Disk(sp, azs, nt=K, dtype="float32", checkpoint_every=200)
             for sp in _inversion_specs(D)]
    d_obs = inversion.observe(disks)
    rng = np.random.default_rng(11)
    x0 = np.concatenate([a for d in disks for a in inversion.isotropic_angles(d.n_grains, rng)])
    inv = inversion.FabricInversion(disks, d_obs, batched=True)
    plain = inversion.FabricInversion(disks, d_obs, batched=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Jp, gp = plain.objective(x0)
    t_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    Jb, gb = inv.objective(x0)
    t_batch = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = inv.run(x0, iterations=I)
    t_run = time.perf_counter() - t0
    errs0, errs = [], []
    for d, (th, ph), (th0, ph0) in zip(disks, inv.split(res["x"]), inv.split(x0)):
        errs.append(inversion.eigen_error(inversion.axes_of(th, ph), d.true_axes))
        errs0.append(inversion.eigen_error(inversion.axes_of(th0, ph0), d.true_axes))
    return {"metric": "L-BFGS fabric inversion, wall time per iteration", "unit": "s/iteration",
            "disks": D, "azimuths": A, "solves_per_evaluation": D * A, "steps": K,
            "grids": [list(d.base["lab"].shape) for d in disks], "grains": [d.n_grains for d in disks],
            "parameters": int(len(x0)), "iterations": res["iterations"], "evaluations": res["evaluations"],
            "s_per_iteration": t_run / max(1, res["iterations"]),
            "per_iteration": res["per_iteration"], "J0": res["J0"], "J": res["J"],
            "evaluation_s_batched": t_batch, "evaluation_s_plain": t_plain,
            "evaluation_speedup": t_plain / t_batch,
            "plain_equals_batched": {"J_rel": abs(Jb - Jp) / abs(Jp),
                                     "grad_rel": float(np.abs(gb - gp).max() / np.abs(gp).max())},
            "eigenvalue_error_start": errs0, "eigenvalue_error_end": errs,
            "config": {"dtype": "f32", "checkpoint_every": 200, "start": "isotropic (seeded)",
                       "observed": "synthetic traces of the true fabric, same solver",
                       "timing": "wall clock per iteration: all batched forward+adjoint evaluations of the line search"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="pefdtd", choices=["pefdtd", "reference"])
    ap.add_argument("--workload", default="disk_prod")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--sweep", type=int, default=0)
    ap.add_argument("--uneven", action="store_true")
    ap.add_argument("--traces", type=int, default=0)
    ap.add_argument("--gradients", type=int, default=0)
    ap.add_argument("--plain-solves", type=int, default=0)
    ap.add_argument("--inversion", type=int, default=0)
    ap.add_argument("--azimuths", type=int, default=36)
    ap.add_argument("--iterations", type=int, default=10)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    K, W = int(args.steps), max(3, int(args.warmup))

    if args.impl == "reference":
        if rank != 0:
            return
        # inputs built on the host only (the labeller's NumPy twin is
        # bit-identical to the device labeller), so that this process loads
        # no library of the CUDA path
        p = _problem(args.workload, nt=max(K, W, 8), use_gpu=False)
        val, n, cores, kind, sample = _cpu_run(p, budget_s=90.0, max_steps=K, warmup=W)
        line = {"metric": "Gcell-updates/s", "value": val, "unit": "Gcell-updates/s",
                "n_gpus": args.gpus, "steps": n, "warmup": W,
                "ms_per_step": int(np.prod(p["lab"].shape)) / (val * 1e9) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": args.workload, "grid": list(p["lab"].shape),
                           "grains": int(p["n_grains"]), "timesteps_per_step": 1},
                "cpu_baseline": {"value": val, "unit": "Gcell-updates/s", "cores": cores,
                                 "cpu_model": _cpu_model(), "kind": kind, "sample": sample},
                "e2e": {"value": val, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if args.sweep:
        if rank == 0:
            print(json.dumps(_sweep(args)), flush=True)
        return
    if args.traces:
        if rank == 0:
            print(json.dumps(_traces(args)), flush=True)
        return
    if args.gradients:
        if rank == 0:
            print(json.dumps(_gradients(args)), flush=True)
        return
    if args.inversion:
        if rank == 0:
            print(json.dumps(_inversion(args)), flush=True)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_total = max(W + K, SPLIT_FROM) + 64
    p = _problem(args.workload, nt=n_total)
    ncell = int(np.prod(p["lab"].shape))
    solve = _device_solve(p, n_total)

    solve.run(0, W)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        ev0.record()
        solve.run(W, W + K)
        ev1.record()
        torch.cuda.synchronize()
    launches = solve.launch_count()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    tr = solve.traces_numpy(W + K)
    finite = bool(np.isfinite(tr).all())

    # per-kernel split for the roofline (events around each launch), taken on
    # a filled wavefield: the first steps after a reset skip most face-density
    # divisions and run faster, so the state is first advanced (untimed) to
    # step SPLIT_FROM when the timed steps ended earlier
    n_done = W + K
    if n_done < SPLIT_FROM:
        solve.run(n_done, SPLIT_FROM)
        n_done = SPLIT_FROM
    ms_s, ms_v = solve.profile(50)
    solve.close()
    peak, peak_kind = _peaks()
    step_ms = ms / K
    value = world * ncell * K / (ms / 1e3) / 1e9
    dominant = "k_stress" if ms_s >= ms_v else "k_velocity"
    dom_ms, dom_b = (ms_s, ALG_BYTES_STRESS) if dominant == "k_stress" else (ms_v, ALG_BYTES_VEL)
    achieved = dom_b * ncell / (dom_ms / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        traffic = tj.get(args.workload, {}).get(dominant)
    except Exception:
        pass
    line = {"metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": args.workload, "grid": list(p["lab"].shape),
                       "grains": int(p["n_grains"]), "h_m": p["h"], "record": p["record"],
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "state 9x4 B/cell = %.0f MB > 126 MB L2, no flush" % (36 * ncell / 1e6)},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_cell": dom_b, "peak_source": peak_kind},
            "roofline_step": {"achieved": ALG_BYTES_STEP * ncell / (step_ms / 1e3) / 1e9,
                              "peak": peak, "unit": "GB/s",
                              "frac": ALG_BYTES_STEP * ncell / (step_ms / 1e3) / 1e9 / peak,
                              "alg_bytes_per_cell": ALG_BYTES_STEP,
                              "kernel_ms": {"k_stress": ms_s, "k_velocity": ms_v},
                              "split_taken_after_steps": n_done, "split_steps": 50},
            "gpu_launches": launches, "traces_finite": finite}
    if rank == 0 and not args.no_e2e:
        line["e2e"] = _e2e(p, K)
    if rank == 0 and not args.no_cpu:
        line["fp64_check"] = _fp64_check(p, int(p["spec"]["nt"]))
    if rank == 0 and not args.no_sweep:
        line["sweep"] = _sweep_compact(SWEEP_STEPS)
    clk_sum = clk.summary()
    if clk_sum is not None:
        line["clocks"] = clk_sum
    if rank == 0 and not args.no_cpu and world == 1:
        val, n, cores, kind, sample = _cpu_run(p, budget_s=20.0, max_steps=200)
        line["cpu_baseline"] = {"value": val, "unit": "Gcell-updates/s", "cores": cores,
                                "cpu_model": _cpu_model(), "kind": kind, "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
