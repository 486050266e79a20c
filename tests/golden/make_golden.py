"""Generate the golden fixtures in tests/golden/ by importing the reference.

Run where the reference tree is present, with PE_REFERENCE_ROOT naming it:
  PE_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py

Every fixture records what the reference itself computes for seeded inputs
(the inputs are stored beside the outputs, so the tests need no reference at
run time):
  coeffs.json        optimised_coeffs / taylor_coeffs / cfl_limit
  tables.npz         material_tables for seeded c-axes; safe_dt_labels
  sponge.npz         sponge_profile volumes; face_density
  wavelets.npz       ricker, hann_tone_burst, pick_peak on a seeded trace
  specimen.npz       DiskSpecimen.build (CPU labeller), build_grid and
                     rotated_grid at two azimuths, sample_watson
  forward_small.npz  fdtd.forward traces (FP64 on CPU, and FP32 through a
                     NumPy stand-in for CuPy) for a small seeded disk, both
                     records, with the inputs that produced them
  sweep_protocol.npz the sweep engine's per-azimuth solver arguments and
                     az{ddd}.npz files on a coarse disk; azimuth orders
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PE_REFERENCE_ROOT")
if not REF or not os.path.isdir(os.path.join(REF, "sim", "core")):
    raise SystemExit("make_golden.py imports the reference: set PE_REFERENCE_ROOT to its checkout "
                     "(the directory holding sim/core/fdtd.py)")
sys.path[:0] = [os.path.join(REF, "sim", "core"), os.path.join(REF, "vendor"),
                os.path.join(REF, "sim", "fw_checks")]


def _numpy_as_cupy():
    """A module that answers to `import cupy` with NumPy, so the reference's
    array path runs its float32 branch on the CPU."""
    m = types.ModuleType("cupy")
    m.__getattr__ = lambda name: getattr(np, name)
    m.asnumpy = np.asarray
    rt = types.SimpleNamespace(getDeviceCount=lambda: 1)
    m.cuda = types.SimpleNamespace(runtime=rt)
    return m


def main():
    import fdtd
    from ringfwi import anisotropy as an
    from ringfwi import sources
    import specimen as spm

    out = {}
    # ---- coefficients
    co = {}
    for order in (2, 4, 6, 8):
        co[f"taylor_{order}"] = list(map(float, fdtd.taylor_coeffs(order)))
    for kh, ms in ((1.6, True), (2.0, True), (1.6, False)):
        co[f"opt_8_{kh}_{ms}"] = list(map(float, fdtd.optimised_coeffs(8, kh_max=kh, multistart=ms)))
    co["opt_4_1.6_True"] = list(map(float, fdtd.optimised_coeffs(4)))
    co["opt_6_1.6_True"] = list(map(float, fdtd.optimised_coeffs(6)))
    co["cfl_8_2.0"] = float(fdtd.cfl_limit(np.array(co["opt_8_2.0_True"])))
    with open(os.path.join(HERE, "coeffs.json"), "w") as f:
        json.dump(co, f, indent=1)

    # ---- material tables
    rng = np.random.default_rng(11)
    axes = rng.normal(size=(300, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    axes[0] = [0, 0, 1]
    axes[1] = [0, 0, -1]
    axes[2] = [1, 0, 0]
    Ct, rho_t = fdtd.material_tables(axes)
    Ct2, rho2 = fdtd.material_tables(axes[:20], c_couplant=1480.0, rho_couplant=1000.0)
    lab = rng.integers(-1, 20, size=(10, 12, 14))
    mats = (lab + 1).astype(np.uint8)
    dt_lab = fdtd.safe_dt_labels(mats, Ct, rho_t, 1e-4, np.array(co["opt_8_2.0_True"]), safety=0.5)
    np.savez_compressed(os.path.join(HERE, "tables.npz"), axes=axes, Ct=Ct, rho_t=rho_t,
                        Ct2=Ct2, rho2=rho2, lab=lab, dt_lab=dt_lab)

    # ---- sponge / face density
    sp1 = fdtd.sponge_profile((20, 24, 30), 6)
    sp2 = fdtd.sponge_profile((9, 40, 7), 5, strength=0.2)
    rho_cell = rng.uniform(300, 917, size=(6, 7, 8))
    fd = np.stack([fdtd.face_density(rho_cell, a) for a in range(3)])
    np.savez_compressed(os.path.join(HERE, "sponge.npz"), sp1=sp1, sp2=sp2, rho_cell=rho_cell, fd=fd)

    # ---- wavelets and picks
    dtw = 2e-8
    rk = fdtd.ricker(2e6, dtw, 800)
    hb = sources.hann_tone_burst(800, dtw, 1e6, n_cycles=3)
    t = np.arange(3000) * dtw
    tr = (np.exp(-((t - 20e-6) / 1e-6) ** 2) * np.sin(2 * np.pi * 2e6 * t)
          + 0.01 * rng.standard_normal(3000))
    pk = fdtd.pick_peak(t, tr, t_lo=10e-6, t_hi=40e-6, dt=dtw)
    pk_hp = fdtd.pick_peak(t, tr, t_lo=10e-6, t_hi=40e-6, dt=dtw, f_lo=0.3e6)
    np.savez_compressed(os.path.join(HERE, "wavelets.npz"), ricker=rk, hann=hb, t=t, tr=tr,
                        pick=np.array(pk[:2]), pick_ok=pk[2], pick_hp=np.array(pk_hp[:2]))

    # ---- specimen (CPU labeller: CuPy absent), grid builders, Watson
    sp = spm.DiskSpecimen(diameter_m=0.012, thickness_m=0.006, n_grains=25, size_cv=0.35,
                          concentration=3.0, spatial_corr=0.0, fabric_axis=(1, 0, 0), seed=7)
    b = sp.build(0.5e-3)
    import coda_convergence as CC
    import rotation_test as RT
    g_lab, nd, m = CC.build_grid(b, 0.4e-3, 4)
    r_lab17, _, _, r_ax17 = RT.rotated_grid(b, 0.4e-3, 4, 17)
    r_lab90, _, _, r_ax90 = RT.rotated_grid(b, 0.4e-3, 4, 90)
    w_rng = np.random.default_rng(3)
    wat = spm.sample_watson(200, (1.0, 0.0, 1.0), 5.0, w_rng)
    wat_g = spm.sample_watson(100, (0.0, 0.0, 1.0), -4.0, w_rng)
    seeds_rng = np.random.default_rng(21)
    seeds = spm.DiskSpecimen._seed_points(5e-3, 3e-3, 40, seeds_rng)
    np.savez_compressed(os.path.join(HERE, "specimen.npz"), labels=b["labels"], axes=b["axes"],
                        seeds=b["seeds"], weights=b["weights"], h=b["h"], grid_lab=g_lab,
                        rot17=r_lab17, rot17_axes=r_ax17, rot90=r_lab90, rot90_axes=r_ax90,
                        watson=wat, watson_girdle=wat_g, seed_pts=seeds)
    # single-raster rotation (seeds rotated, shortlist labeller) and a
    # neighbour-smoothed fabric
    s_lab, _, _, s_ax = RT.rotated_grid(b, 0.4e-3, 4, 33, single_raster=True)
    sp2 = spm.DiskSpecimen(diameter_m=0.010, thickness_m=0.005, n_grains=30, size_cv=0.5,
                           concentration=-2.0, spatial_corr=0.4, fabric_axis=(0, 1, 1), seed=11)
    b2 = sp2.build(0.5e-3)
    np.savez_compressed(os.path.join(HERE, "specimen2.npz"), rot33_single=s_lab, rot33_axes=s_ax,
                        labels=b2["labels"], axes=b2["axes"], seeds=b2["seeds"],
                        weights=b2["weights"])

    # ---- forward traces on a small seeded disk
    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import make_small
    p = make_small(nt=160, shape=(22, 26, 30), n_grains=10, sponge=4)
    lab = p["lab"]
    C, rho = an.polycrystal_stiffness_3d(lab, p["axes"], c_couplant=1500.0, rho_couplant=300.0)
    res = dict(lab=lab.astype(np.int16), axes=p["axes"], h=p["h"], dt=p["dt"], nt=p["nt"],
               coeffs=p["coeffs"], wavelet=p["wavelet"], sponge=p["sponge"],
               src=np.array([q for q, _ in p["src_pts"]]), w=p["src_pts"][0][1])
    recs = p["rec_groups"]
    for record in ("pressure", "vz"):
        tr64 = fdtd.forward(C, rho, p["h"], p["dt"], p["nt"], p["src_pts"], p["wavelet"], recs,
                            coeffs=p["coeffs"], sponge_width=p["sponge"], device="cpu",
                            record=record)
        sys.modules["cupy"] = _numpy_as_cupy()
        try:
            tr32 = fdtd.forward(C, rho, p["h"], p["dt"], p["nt"], p["src_pts"], p["wavelet"],
                                recs, coeffs=p["coeffs"], sponge_width=p["sponge"], device="gpu",
                                record=record)
        finally:
            del sys.modules["cupy"]
        res[f"{record}_f64"] = tr64
        res[f"{record}_f32"] = tr32
    np.savez_compressed(os.path.join(HERE, "forward_small.npz"), **res)
    adjoint_compat()
    sweep_protocol()
    print("golden fixtures written to", HERE)


SWEEP_CFG = dict(f0_mhz=0.5, ppw=6.0, az_start=0, az_stop=360, az_step=45, diameter_mm=80.0,
                 thickness_mm=10.0, n_grains=12, sponge=10, seed=5)


def sweep_protocol():
    """The reference sweep engine (sim/pipeline/sweep_runner.py) run on a
    coarse 80 mm disk with a NumPy stand-in for CuPy (so its exact all-seeds
    labeller runs) and forward_fused_labels replaced by a recorder that
    returns tests/helpers.synthetic_echo: every solver argument it passes
    per azimuth, and the az{ddd}.npz files it writes."""
    import hashlib
    import shutil
    import tempfile
    sys.path.insert(0, os.path.join(REF, "sim", "pipeline"))
    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import synthetic_echo
    cp = _numpy_as_cupy()
    cp.cuda.runtime.getDeviceProperties = lambda i: {"name": b"numpy"}
    sys.modules["cupy"] = cp
    import sweep_runner as SR
    import fdtd as F
    calls = {}

    def recorder(lab, axes, h, dt, nt, src_pts, wavelet, rec_groups, order=8, coeffs=None,
                 sponge_width=0, damp_mask=None, progress=None, **kw):
        az = len(calls)
        calls[az] = dict(lab=lab, axes=axes, h=h, dt=dt, nt=nt, src=src_pts, wav=wavelet,
                         rec=rec_groups, order=order, coeffs=coeffs, sponge=sponge_width,
                         dm=damp_mask)
        if progress is not None:
            progress(0.0)
        return synthetic_echo(nt, dt, 0.5e6)[:, None]
    orig = F.forward_fused_labels
    F.forward_fused_labels = recorder
    tmp = tempfile.mkdtemp()
    try:
        SR.SWEEPS = tmp
        SR.create("fx", **SWEEP_CFG)
        cfg = SR.load("fx")
        order = SR.azimuths(cfg)
        SR.run(cfg)
        res = dict(order=np.array(order))
        sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
        for i, az in enumerate(order):
            c = calls[i]
            with np.load(os.path.join(tmp, "fx", f"az{az:03d}.npz")) as z:
                for k in z.files:
                    res[f"{az}_file_{k}"] = z[k]
            res[f"{az}_lab_shape"] = np.array(c["lab"].shape)
            res[f"{az}_lab_sha"] = sha(np.asarray(c["lab"], np.int32))
            res[f"{az}_dm_sha"] = sha(np.asarray(c["dm"], np.float32))
            res[f"{az}_wav_sha"] = sha(np.asarray(c["wav"], np.float64))
            res[f"{az}_axes"] = np.asarray(c["axes"])
            res[f"{az}_dt"] = c["dt"]
            res[f"{az}_nt"] = c["nt"]
            res[f"{az}_src"] = np.array([p for p, _ in c["src"]])
            res[f"{az}_w"] = c["src"][0][1]
            res[f"{az}_coeffs"] = np.asarray(c["coeffs"])
        with open(os.path.join(tmp, "fx", "status.json")) as f:
            res["final_phase"] = json.load(f)["phase"]
        orders = {}
        for n in range(0, 70):
            orders[f"bitrev_{n}"] = np.array(SR._bit_reversed_order(n), np.int64)
        for start, stop, step, mode in ((0, 360, 1, "progressive"), (10, 350, 7, "progressive"),
                                        (0, 180, 4, "progressive"), (0, 360, 5, "sequential")):
            c2 = dict(az_start=start, az_stop=stop, az_step=step, sweep_order=mode)
            orders[f"az_{start}_{stop}_{step}_{mode}"] = np.array(SR.azimuths(c2), np.int64)
        res.update(orders)
        np.savez_compressed(os.path.join(HERE, "sweep_protocol.npz"), **res)
    finally:
        F.forward_fused_labels = orig
        del sys.modules["cupy"]
        shutil.rmtree(tmp)


def adjoint_compat():
    """The reference's own gradient (vendor/ringfwi/axisfield.py:123-161 over
    vendor/ringfwi/elastic3d.py:348-463) on a small matched problem: order 2,
    no damping, pressure record, uniform density 917 (so face and cell
    density agree), explosive source, one receiver group. Stores the inputs,
    the observed traces, J and the per-grain (colatitude, azimuth) gradients
    (per-voxel gradients summed over each grain)."""
    from ringfwi import anisotropy as an
    from ringfwi import axisfield as af
    from ringfwi import elastic3d as e3
    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import make_small
    p = make_small(nt=60, shape=(16, 20, 20), n_grains=6, sponge=0, seed=3)
    lab = p["lab"]
    n_g = int(lab.max()) + 1
    rng = np.random.default_rng(5)
    theta = rng.uniform(0.2, 1.3, n_g)
    phi = rng.uniform(-3.0, 3.0, n_g)
    theta_obs = theta + rng.normal(0, 0.15, n_g)
    phi_obs = phi + rng.normal(0, 0.15, n_g)
    mask = lab >= 0
    base6 = an.ti_stiffness_6(**an.ICE_MATERIAL)
    K = 917.0 * 1500.0 ** 2
    fl = np.zeros((6, 6))
    fl[:3, :3] = K
    Cbg = {k: np.full(lab.shape, fl[int(k[1]) - 1, int(k[2]) - 1]) for k in af.KEYS21}
    h = p["h"]
    dt = 0.4 * h / (np.sqrt(3.0) * 4100.0)
    nt = 60
    wav = sources_hann(nt, dt)
    pts = [tuple(q) for q, _ in p["src_pts"]]
    w = 1.0 / len(pts)
    src_pts = [[(q, w) for q in pts]]
    recs = [(pts, [w] * len(pts))]

    def maps(th, ph):
        cm = np.zeros(lab.shape)
        am = np.zeros(lab.shape)
        cm[mask] = th[lab[mask]]
        am[mask] = ph[lab[mask]]
        return cm, am

    co, ao = maps(theta_obs, phi_obs)
    Cobs, rho = af.build_maps(co, ao, mask, base6, Cbg, 917.0, 917.0)
    dobs, _ = e3._grad_forward(Cobs, rho, h, dt, nt, None, wav, None, src_pts=src_pts[0],
                               rec_groups=recs)
    cm, am = maps(theta, phi)
    J, g_t, g_p = af.misfit_and_gradient_axes(cm, am, mask, base6, Cbg, 917.0, 917.0, h, dt, nt,
                                              src_pts, wav, recs, dobs[None])
    gt = np.array([g_t[lab == g].sum() for g in range(n_g)])
    gp = np.array([g_p[lab == g].sum() for g in range(n_g)])
    np.savez_compressed(os.path.join(HERE, "adjoint_compat.npz"), lab=lab.astype(np.int16),
                        theta=theta, phi=phi, h=h, dt=dt, nt=nt, wavelet=wav,
                        pts=np.array(pts), dobs=dobs, J=J, g_theta=gt, g_phi=gp)


def sources_hann(nt, dt):
    from ringfwi import sources
    return sources.hann_tone_burst(nt, dt, 2.0e6, n_cycles=2)


if __name__ == "__main__":
    main()
