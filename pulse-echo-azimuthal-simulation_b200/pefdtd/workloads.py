"""Seeded synthetic pulse-echo problems: ice disks in a fluid couplant.

Two named workloads, with the shapes, sizes and value distributions of the
benchmark configurations this solver is measured on:

  disk_small   64 x 96 x 96 cells at h = 0.2 mm; disk 18 mm x 10 mm with 50
               Voronoi grains; Watson kappa = 5 about an axis 30 deg from z;
               1 MHz 3-cycle Hann burst; 2000 steps; 20-cell sponge.
  disk_prod    160 x 256 x 256 cells at h = 0.1 mm; disk 25 mm x 10 mm with
               500 Voronoi grains; girdle fabric (great circle tilted 20 deg
               from horizontal, 10 deg Gaussian scatter); 2.25 MHz 5-cycle
               Hann burst; 6000 steps; 32-cell sponge.

Both: CFL safety 0.5 on the discrete grid speed (safe_dt_labels), order-8
dispersion-optimised coefficients (kh_max 2.0, the reference's production
band), fluid couplant c = 1500 m/s, rho = 300 kg/m^3 (the reference's row 0),
a 6 mm-aperture transducer on the top ice face (the first ice z-plane) that
is both the explosive source and the receiver (weights 1/N), z-velocity
recorded. The disk sits inside the sponge, so traces are recorded with the
dense path's end-of-step damping (damped_record=True).

Labels come from an exact power-diagram argmin (pure Voronoi: weights 0) over
seeds drawn uniformly in the cylinder, empty cells dropped; the grid is built
directly in solver order and centred.
"""
from __future__ import annotations

import numpy as np

from .coeffs import optimised_coeffs
from .damping import safe_dt_labels
from .materials import material_tables
from .specimen import (label_cylinder, label_cylinder_numpy, relabel_contiguous,
                       sample_great_circle, sample_watson, seed_points)
from .wavelets import hann_tone_burst

WORKLOADS = {
    "disk_small": dict(shape=(64, 96, 96), h=0.2e-3, diameter=18e-3, height=10e-3,
                       n_grains=50, fabric=("watson", 30.0, 5.0), f0=1.0e6, n_cycles=3,
                       nt=2000, sponge=20, aperture=6e-3, seed=1),
    "disk_prod": dict(shape=(160, 256, 256), h=0.1e-3, diameter=25e-3, height=10e-3,
                      n_grains=500, fabric=("girdle", 20.0, 10.0), f0=2.25e6, n_cycles=5,
                      nt=6000, sponge=32, aperture=6e-3, seed=2),
}


def disk_labels(shape, h, diameter, height, n_grains, seed, use_gpu=None):
    """(lab (nz, ny, nx) int32 with -1 outside, n_realised, rng after seeding)."""
    rng = np.random.default_rng(seed)
    R = diameter / 2
    nd = int(round(diameter / h))
    nzd = int(round(height / h))
    nz, ny, nx = shape
    if nd > min(ny, nx) or nzd > nz:
        raise ValueError("disk does not fit the grid")
    seeds = seed_points(R, height, n_grains, rng)
    c = (np.arange(nd) - (nd - 1) / 2) * h
    zc = (np.arange(nzd) - (nzd - 1) / 2) * h
    if use_gpu is None:
        try:
            import torch
            use_gpu = torch.cuda.is_available()
        except Exception:
            use_gpu = False
    if use_gpu:
        raw = label_cylinder(c, c, zc, R, seeds).cpu().numpy()
    else:
        raw = label_cylinder_numpy(c, c, zc, R, seeds)
    core, keep = relabel_contiguous(raw)
    lab = np.full(shape, -1, np.int32)
    oz, oy, ox = (nz - nzd) // 2, (ny - nd) // 2, (nx - nd) // 2
    lab[oz:oz + nzd, oy:oy + nd, ox:ox + nd] = core
    return lab, len(keep), rng


def top_probe(lab, h, aperture):
    """Cells of the first ice z-plane within aperture/2 of the disk axis."""
    nz, ny, nx = lab.shape
    ice_z = np.nonzero((lab >= 0).any(axis=(1, 2)))[0]
    iz = int(ice_z[0])
    r = aperture / 2
    yc, xc = (ny - 1) / 2, (nx - 1) / 2
    Y, X = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    inside = (((Y - yc) * h) ** 2 + ((X - xc) * h) ** 2 <= r * r) & (lab[iz] >= 0)
    iy, ix = np.nonzero(inside)            # row-major: the order of the (iy, ix) loop
    return [(iz, int(a), int(b)) for a, b in zip(iy, ix)]


def make_problem(name_or_spec, nt=None, use_gpu=None, kh_max=2.0):
    """All inputs of one solve as a dict (numpy arrays, host side)."""
    spec = dict(WORKLOADS[name_or_spec]) if isinstance(name_or_spec, str) else dict(name_or_spec)
    lab, n_real, rng = disk_labels(spec["shape"], spec["h"], spec["diameter"], spec["height"],
                                   spec["n_grains"], spec["seed"], use_gpu=use_gpu)
    kind, a, b = spec["fabric"]
    if kind == "watson":
        t = np.radians(a)
        axes = sample_watson(n_real, (np.sin(t), 0.0, np.cos(t)), b, rng)
    elif kind == "girdle":
        axes = sample_great_circle(n_real, a, b, rng)
    else:
        raise ValueError(kind)
    Ct, rho_t = material_tables(axes)
    mats = (lab + 1).astype(np.uint16)
    coeffs = optimised_coeffs(8, kh_max=kh_max)
    h = spec["h"]
    dt = safe_dt_labels(mats, Ct, rho_t, h, coeffs, safety=0.5)
    nt = int(spec["nt"] if nt is None else nt)
    wav = hann_tone_burst(nt, dt, spec["f0"], n_cycles=spec["n_cycles"])
    pts = top_probe(lab, h, spec["aperture"])
    w = 1.0 / len(pts)
    return dict(name=name_or_spec if isinstance(name_or_spec, str) else "custom", spec=spec,
                lab=lab, axes=axes, n_grains=n_real, Ct=Ct, rho_t=rho_t, mats=mats, h=h, dt=dt,
                nt=nt, coeffs=coeffs, wavelet=wav, src_pts=[(p, w) for p in pts],
                rec_groups=[(pts, np.full(len(pts), w))], sponge=spec["sponge"],
                record="vz")


def bottom_echo_window(p):
    """Where the disk's bottom-face echo must be picked, for a problem from
    make_problem: (t_lo, win_lo, win_hi) in seconds.

    The probe sits on the top ice face, so the echo travels 2 x height through
    ice. Vertical qP speeds of the hexagonal ice lie between sqrt(C11 / rho)
    (c-axis horizontal) and sqrt(C33 / rho) (c-axis vertical); the window
    spans those round trips with a 5 % margin, plus the burst length for the
    echo's envelope. t_lo, the start of the pick's search, lies halfway
    between the end of the transmitted burst and the earliest echo, so the
    transmitted burst is outside the search."""
    from .materials import ICE
    spec = p["spec"]
    H = float(spec["height"])
    c_fast = np.sqrt(ICE["C33"] / ICE["rho"])
    c_slow = np.sqrt(ICE["C11"] / ICE["rho"])
    burst = spec["n_cycles"] / spec["f0"]
    win_lo = 2.0 * H / (1.05 * c_fast)
    win_hi = 2.0 * H / (0.95 * c_slow) + burst
    return 0.5 * (burst + win_lo), win_lo, win_hi
