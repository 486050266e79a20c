"""Absorbing sponge, face density and the stable time step.

Restates sim/core/fdtd.py:211-233 (sponge_profile), :987-1038 (face_density,
max_grid_speed, safe_dt), :1560-1577 (absorption_mask) and :1606-1615
(safe_dt_labels).

The kernels never read a damping volume when only the sponge is active: the
sponge is a product of three 1D tapers, so they take the three f32 profiles
and form fl(fl(pz * py) * px) per cell, which is bit-for-bit the f32 volume
the reference multiplies together axis by axis (z, then y, then x).
"""
from __future__ import annotations

import numpy as np


def sponge_axis_profiles(shape, width, strength=0.09):
    """Three f32 1D tapers (z, y, x) whose product is the sponge volume."""
    out = []
    for n in shape:
        prof = np.ones(n)
        w = min(int(width), n // 2)
        if width > 0 and w > 0:
            t = np.arange(w) / w
            taper = np.exp(-strength * (1.0 - t) ** 2 * w)
            prof[:w] = taper
            prof[n - w:] = taper[::-1]
        out.append(prof.astype(np.float32))
    return tuple(out)


def sponge_profile(shape, width, strength=0.09):
    """Multiplicative per-step damping volume (f32), 1 in the interior."""
    d = np.ones(shape, np.float32)
    if width <= 0:
        return d
    pz, py, px = sponge_axis_profiles(shape, width, strength)
    d *= pz.reshape(-1, 1, 1)
    d *= py.reshape(1, -1, 1)
    d *= px.reshape(1, 1, -1)
    return d


def face_density(rho, ax):
    """Arithmetic mean of the two cells a velocity node straddles along ``ax``;
    the last slice keeps its own value."""
    a = np.asarray(rho, float)
    m = np.empty_like(a)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[ax] = slice(0, -1)
    hi[ax] = slice(1, None)
    m[tuple(lo)] = 0.5 * (a[tuple(lo)] + a[tuple(hi)])
    last = [slice(None)] * 3
    last[ax] = slice(-1, None)
    m[tuple(last)] = a[tuple(last)]
    return m


def max_grid_speed(C, rho):
    """Worst discrete speed sqrt(max(C11,C22,C33) / min(rho, face rho))."""
    rho_h = np.asarray(rho, float)
    Cmax = np.maximum.reduce([np.broadcast_to(np.asarray(C[k], float), rho_h.shape)
                              for k in ("C11", "C22", "C33")])
    rmin = rho_h.copy()
    for ax in range(3):
        np.minimum(rmin, face_density(rho_h, ax), out=rmin)
    return float(np.sqrt(Cmax / rmin).max())


def safe_dt(C, rho, h, coeffs, safety=0.85):
    from .coeffs import cfl_limit
    return safety * cfl_limit(np.asarray(coeffs, float)) * h / max_grid_speed(C, rho)


def safe_dt_labels(mats, Ct, rho_t, h, coeffs, safety=0.85):
    """safe_dt from material indices and tables, no per-cell stiffness."""
    from .coeffs import cfl_limit
    Ct = np.asarray(Ct).reshape(-1, 36)
    diag = Ct[:, [0, 7, 14]].max(axis=1)
    Cmax = diag[mats]
    rho = np.asarray(rho_t)[mats].astype(float)
    rmin = rho.copy()
    for ax in range(3):
        np.minimum(rmin, face_density(rho, ax), out=rmin)
    vmax = float(np.sqrt(Cmax / rmin).max())
    return safety * cfl_limit(np.asarray(coeffs, float)) * h / vmax


def absorption_mask(lab, alpha_np_m, c_ref, dt):
    """Per-step amplitude factor exp(-alpha c dt) in ice cells, 1 in fluid."""
    lab = np.asarray(lab)
    f = float(np.exp(-alpha_np_m * c_ref * dt))
    m = np.ones(lab.shape, np.float32)
    m[lab >= 0] = f
    return m


def fluid_damp_mask(lab, fluid_damp=0.02):
    """exp(-fluid_damp * distance-to-ice) in the fluid, 1 in ice — the mask
    the reference's drivers pass as ``damp_mask``
    (sim/core/validate_labels.py:51-52, sim/pipeline/sweep_runner.py:340-341)."""
    from scipy import ndimage
    dist = ndimage.distance_transform_edt((np.asarray(lab) < 0).astype(np.float32))
    return np.exp(-fluid_damp * dist).astype(np.float32)
