"""Polycrystalline ice-disk label volumes and c-axis fabrics.

Restates the reference's specimen machinery where it fixes integer results:
  seed points in a cylinder     sim/core/specimen.py:281-288 (_seed_points)
  power-diagram labelling       sim/core/specimen.py:298-337 (_label_grid_gpu:
                                exact all-seeds argmin in float64, distance
                                ((x-sx)^2 + (y-sy)^2) - w + (z-sz)^2, first
                                index on ties, -1 outside x^2 + y^2 <= R^2)
  drop empty cells, relabel     sim/core/specimen.py:238-247
  Watson fabric                 sim/core/specimen.py:45-69 (sample_watson)
  orientation tensor            sim/core/specimen.py:146-155
  solver grid from a specimen   sim/fw_checks/coda_convergence.py:40-53
                                (build_grid) and sim/core/rotation_test.py:60-137
                                (rotated_grid)
The label volume here is produced directly in solver order (z, y, x); the
reference builds (x, y, z) and transposes, which is the same map.

``label_cylinder`` runs on the GPU through the C ABI (pe_label_cylinder);
``label_cylinder_numpy`` is the same arithmetic in NumPy for small grids.
"""
from __future__ import annotations

import numpy as np

from .materials import rotation_z_to


def seed_points(R, thickness, n, rng):
    """n points uniform in the cylinder r <= R, |z| <= thickness/2 (rejection
    from the unit cube, 3n candidates per round)."""
    pts = []
    while len(pts) < n:
        p = rng.uniform(-1, 1, (n * 3, 3))
        pts.extend(p[(p[:, 0] ** 2 + p[:, 1] ** 2) <= 1.0].tolist())
    s = np.array(pts[:n])
    s[:, :2] *= R
    s[:, 2] *= thickness / 2
    return s


def label_cylinder_numpy(xs, ys, zs, R, seeds, weights=None, chunk=1 << 16):
    """(nz, ny, nx) int32 power-diagram labels; -1 outside the cylinder."""
    xs, ys, zs = (np.asarray(a, float) for a in (xs, ys, zs))
    seeds = np.asarray(seeds, float)
    w = np.zeros(len(seeds)) if weights is None else np.asarray(weights, float)
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # (ny, nx)
    inside = (X ** 2 + Y ** 2) <= R ** 2
    P = np.stack([X[inside], Y[inside]], axis=1)
    out = np.full((len(zs), len(ys), len(xs)), -1, np.int32)
    lab_plane = np.empty(len(P), np.int32)
    for iz, z in enumerate(zs):
        dz2 = (z - seeds[:, 2]) ** 2
        for a in range(0, len(P), chunk):
            p = P[a:a + chunk]
            d = (((p[:, None, :] - seeds[None, :, :2]) ** 2).sum(-1) - w[None, :]) + dz2[None, :]
            lab_plane[a:a + chunk] = d.argmin(axis=1)
        plane = out[iz]
        plane[inside] = lab_plane
    return out


def label_cylinder(xs, ys, zs, R, seeds, weights=None, device=None):
    """GPU power-diagram labels, bit-identical to label_cylinder_numpy."""
    from . import _capi
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("label_cylinder runs on a CUDA device; use label_cylinder_numpy on CPU")
    xs, ys, zs = (np.ascontiguousarray(a, np.float64) for a in (xs, ys, zs))
    seeds = np.ascontiguousarray(seeds, np.float64).reshape(-1, 3)
    w = (np.zeros(len(seeds)) if weights is None else np.ascontiguousarray(weights, np.float64))
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    out = torch.empty((len(zs), len(ys), len(xs)), dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        _capi.check(_capi.lib().pe_label_cylinder(
            _capi.ptr(xs), len(xs), _capi.ptr(ys), len(ys), _capi.ptr(zs), len(zs), float(R) ** 2,
            _capi.ptr(seeds), _capi.ptr(w), len(seeds), out.data_ptr(),
            _capi.C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
        torch.cuda.current_stream(dev).synchronize()
    return out


def relabel_contiguous(raw):
    """Drop seeds that own no cell and renumber the rest 0..n-1 in seed order;
    returns (labels, kept seed indices)."""
    raw = np.asarray(raw)
    inside = raw >= 0
    keep = np.unique(raw[inside])
    remap = np.full(int(raw.max()) + 1 if inside.any() else 1, -1, np.int32)
    remap[keep] = np.arange(len(keep), dtype=np.int32)
    lab = np.full(raw.shape, -1, np.int32)
    lab[inside] = remap[raw[inside]]
    return lab, keep


def sample_watson(n, axis, kappa, rng):
    """Watson-distributed unit axes about ``axis`` (kappa > 0 clustered,
    kappa < 0 girdle, 0 uniform)."""
    axis = np.asarray(axis, float)
    axis = axis / np.linalg.norm(axis)
    if abs(kappa) < 1e-9:
        v = rng.normal(size=(n, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)
    t = np.empty(n)
    got = 0
    while got < n:
        u = rng.uniform(-1, 1, n)
        keep = rng.uniform(0, 1, n) < np.exp(kappa * (u ** 2 - (1 if kappa > 0 else 0)))
        k = u[keep][: n - got]
        t[got:got + k.size] = k
        got += k.size
    phi = rng.uniform(0, 2 * np.pi, n)
    s = np.sqrt(np.clip(1 - t ** 2, 0, None))
    local = np.stack([s * np.cos(phi), s * np.sin(phi), t], axis=1)
    return local @ rotation_z_to(axis).T


def sample_great_circle(n, tilt_deg, scatter_deg, rng):
    """Girdle fabric: axes uniform on a great circle whose plane is tilted
    ``tilt_deg`` from horizontal (about y), each then tipped by a Gaussian
    angle of std ``scatter_deg`` about a random perpendicular. Not a
    reference generator; the seeded construction of this module."""
    t = np.radians(tilt_deg)
    e1 = np.array([np.cos(t), 0.0, -np.sin(t)])
    e2 = np.array([0.0, 1.0, 0.0])
    phi = rng.uniform(0, 2 * np.pi, n)
    a = np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2
    psi = np.radians(scatter_deg) * rng.standard_normal(n)
    r = rng.normal(size=(n, 3))
    r -= (r * a).sum(1, keepdims=True) * a
    r /= np.linalg.norm(r, axis=1, keepdims=True)
    out = np.cos(psi)[:, None] * a + np.sin(psi)[:, None] * r
    return out / np.linalg.norm(out, axis=1, keepdims=True)


def orientation_tensor(axes):
    a = np.asarray(axes, float)
    a = a / np.linalg.norm(a, axis=1, keepdims=True)
    T = (a[:, :, None] * a[:, None, :]).mean(axis=0)
    w, V = np.linalg.eigh(T)
    o = np.argsort(w)[::-1]
    return w[o], V[:, o]


def build_grid(labels_xyz, h_spec, h, sponge):
    """Nearest-sample a specimen label volume (x, y, z) at spacing h_spec onto
    the solver grid at spacing h and pad by sponge + 3 fluid cells; returns
    (lab (nz, ny, nx), nd, m)."""
    labels = np.asarray(labels_xyz)
    nx_s, _, nz_s = labels.shape
    D = nx_s * h_spec
    nd = int(round(D / h))
    ndz = int(round(nz_s * h_spec / h))
    gx = np.clip((np.arange(nd) + 0.5) * h / h_spec, 0, nx_s - 1).astype(int)
    gz = np.clip((np.arange(ndz) + 0.5) * h / h_spec, 0, nz_s - 1).astype(int)
    core = labels[np.ix_(gx, gx, gz)].transpose(2, 1, 0).astype(np.int32)
    m = sponge + 3
    nz, nx = ndz + 2 * m, nd + 2 * m
    lab = np.full((nz, nx, nx), -1, np.int32)
    lab[m:m + ndz, m:m + nd, m:m + nd] = core
    return lab, nd, m


def rotated_grid(labels_xyz, axes, h_spec, h, sponge, rot_deg):
    """Solver grid of the specimen rotated by -rot_deg about z (nearest
    resample with np.rint), with the c-axes rotated the same way
    (axes @ R); returns (lab, nd, m, axes_rot)."""
    labels = np.asarray(labels_xyz)
    nx_s, _, nz_s = labels.shape
    D = nx_s * h_spec
    nd = int(round(D / h))
    ndz = int(round(nz_s * h_spec / h))
    a = np.radians(rot_deg)
    ca, sa = np.cos(a), np.sin(a)
    u = (np.arange(nd) + 0.5) * h - D / 2.0
    X, Y = np.meshgrid(u, u, indexing="ij")
    Xr = ca * X - sa * Y
    Yr = sa * X + ca * Y
    gi = np.rint(Xr / h_spec + (nx_s - 1) / 2.0).astype(int)
    gj = np.rint(Yr / h_spec + (nx_s - 1) / 2.0).astype(int)
    ok = (gi >= 0) & (gi < nx_s) & (gj >= 0) & (gj < nx_s)
    gi, gj = np.clip(gi, 0, nx_s - 1), np.clip(gj, 0, nx_s - 1)
    gz = np.clip((np.arange(ndz) + 0.5) * h / h_spec, 0, nz_s - 1).astype(int)
    core = np.where(ok[:, :, None], labels[gi, gj][:, :, gz], -1).astype(np.int32)
    core = core.transpose(2, 1, 0)
    m = sponge + 3
    nz, nx = ndz + 2 * m, nd + 2 * m
    lab = np.full((nz, nx, nx), -1, np.int32)
    lab[m:m + ndz, m:m + nd, m:m + nd] = core
    R = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])
    return lab, nd, m, np.asarray(axes, float) @ R
