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

import os

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


def label_cylinder_numpy(xs, ys, zs, R, seeds, weights=None, chunk=1 << 13):
    """(nz, ny, nx) int32 power-diagram labels; -1 outside the cylinder."""
    xs, ys, zs = (np.asarray(a, float) for a in (xs, ys, zs))
    seeds = np.asarray(seeds, float)
    w = np.zeros(len(seeds)) if weights is None else np.asarray(weights, float)
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # (ny, nx)
    inside = (X ** 2 + Y ** 2) <= R ** 2
    P = np.stack([X[inside], Y[inside]], axis=1)
    out = np.full((len(zs), len(ys), len(xs)), -1, np.int32)

    def plane(iz):
        # each plane is independent: the same element-wise arithmetic whichever
        # thread runs it (NumPy releases the GIL inside the array operations)
        dz2 = (zs[iz] - seeds[:, 2]) ** 2
        lab_plane = np.empty(len(P), np.int32)
        for a in range(0, len(P), chunk):
            p = P[a:a + chunk]
            d = (((p[:, None, :] - seeds[None, :, :2]) ** 2).sum(-1) - w[None, :]) + dz2[None, :]
            lab_plane[a:a + chunk] = d.argmin(axis=1)
        out[iz][inside] = lab_plane

    n_threads = max(1, min(len(zs), os.cpu_count() or 1))
    if n_threads == 1:
        for iz in range(len(zs)):
            plane(iz)
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(n_threads) as ex:
            list(ex.map(plane, range(len(zs))))
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


def assign_shortlist(P, seeds, weights, k=12):
    """Laguerre assignment through the k Euclidean-nearest seeds (the CPU
    labeller of sim/core/specimen.py:339-351; exact while the weight spread
    is modest). Returns int16 seed indices."""
    from scipy.spatial import cKDTree
    k = min(k, len(seeds))
    _, idx = cKDTree(seeds).query(P, k=k, workers=-1)
    idx = np.atleast_2d(idx.T).T
    d2 = ((P[:, None, :] - seeds[idx]) ** 2).sum(-1) - weights[idx]
    return idx[np.arange(len(P)), d2.argmin(1)].astype(np.int16)


def adjacency(labels):
    """Grain adjacency {label: set(neighbour labels)} over face neighbours."""
    adj = {}
    for ax in range(3):
        a = np.take(labels, np.arange(labels.shape[ax] - 1), axis=ax)
        b = np.take(labels, np.arange(1, labels.shape[ax]), axis=ax)
        m = (a != b) & (a >= 0) & (b >= 0)
        for u, v in np.unique(np.stack([a[m], b[m]], 1), axis=0):
            adj.setdefault(int(u), set()).add(int(v))
            adj.setdefault(int(v), set()).add(int(u))
    return adj


def renormalise_fabric(axes, target_a1, n_iter=60):
    """Rescale every axis's angle from the dominant eigenvector until the
    largest orientation-tensor eigenvalue is back at target_a1."""
    w, V = orientation_tensor(axes)
    if abs(w[0] - target_a1) < 1e-4:
        return axes
    e1 = V[:, 0]
    sgn = np.sign(axes @ e1)
    sgn[sgn == 0] = 1.0
    a = axes * sgn[:, None]
    cos = np.clip(a @ e1, -1.0, 1.0)
    psi = np.arccos(cos)
    perp = a - cos[:, None] * e1[None, :]
    pn = np.linalg.norm(perp, axis=1, keepdims=True)
    perp = np.divide(perp, np.maximum(pn, 1e-12), out=np.zeros_like(perp), where=pn > 1e-12)

    def rebuild(k):
        p2 = np.minimum(psi * k, np.pi / 2)
        return np.cos(p2)[:, None] * e1[None, :] + np.sin(p2)[:, None] * perp

    lo, hi = 0.0, 6.0
    for _ in range(n_iter):
        k = 0.5 * (lo + hi)
        if orientation_tensor(rebuild(k))[0][0] > target_a1:
            lo = k
        else:
            hi = k
    out = rebuild(0.5 * (lo + hi))
    return out / np.linalg.norm(out, axis=1, keepdims=True)


class DiskSpecimen:
    """Laguerre-polycrystal ice disk with a Watson c-axis fabric.

    Same controls, random stream and results as the reference's
    ``DiskSpecimen`` (sim/core/specimen.py:166-279): the seed count and
    Laguerre weight scale are calibrated on Monte-Carlo points (12-nearest
    shortlist) to the requested grain-size CV, the grid is then labelled with
    the exact all-seeds power argmin (on the GPU when one is available, else
    with the shortlist, as the reference falls back), empty cells are dropped,
    c-axes are Watson-sampled and optionally smoothed toward neighbours.
    """

    def __init__(self, diameter_m=100e-3, thickness_m=35e-3, n_grains=400, size_cv=0.35,
                 concentration=4.0, spatial_corr=0.0, fabric_axis=(0.0, 0.0, 1.0), seed=7):
        self.diameter_m, self.thickness_m, self.n_grains = diameter_m, thickness_m, n_grains
        self.size_cv, self.concentration, self.spatial_corr = size_cv, concentration, spatial_corr
        self.fabric_axis, self.seed = tuple(fabric_axis), seed

    @staticmethod
    def _mc_points(R, thickness, n, rng):
        p = rng.uniform(-1, 1, (int(n * 1.4), 3))
        p = p[(p[:, 0] ** 2 + p[:, 1] ** 2) <= 1.0][:n]
        p[:, :2] *= R
        p[:, 2] *= thickness / 2
        return p

    def calibrate(self, rng):
        R = self.diameter_m / 2
        mc = self._mc_points(R, self.thickness_m, 400000, rng)
        base = (R / self.n_grains ** (1 / 3)) ** 2
        sigma = np.sqrt(np.log(1 + self.size_cv ** 2))
        n_seed = self.n_grains
        for outer in range(4):
            seeds = seed_points(R, self.thickness_m, n_seed, rng)
            radii = rng.lognormal(-0.5 * sigma ** 2, sigma, n_seed)
            wshape = base * (radii ** 2 - 1.0)
            lo, hi, scale = 0.0, 8.0, 0.0
            for _ in range(20):
                trial = 0.5 * (lo + hi)
                cnt = np.bincount(assign_shortlist(mc, seeds, trial * wshape), minlength=n_seed).astype(float)
                live = cnt[cnt > 0]
                cv = (live ** (1 / 3)).std() / (live ** (1 / 3)).mean()
                if cv < self.size_cv:
                    lo = trial
                else:
                    hi = trial
                scale = trial
            n_live = int((np.bincount(assign_shortlist(mc, seeds, scale * wshape),
                                      minlength=n_seed) > 0).sum())
            if n_live >= self.n_grains or outer == 3:
                break
            n_seed = int(np.ceil(n_seed * self.n_grains / max(n_live, 1)))
        return seeds, scale * wshape, n_seed

    def build(self, h, use_gpu=None, labeller=None):
        """Label volume (x, y, z), c-axes, seeds and weights at spacing h.
        ``labeller``: "gpu" (exact, pe_label_cylinder), "exact" (the same
        argmin in NumPy) or "shortlist" (the reference's CPU fallback);
        default "gpu" when a CUDA device is present, else "shortlist"."""
        rng = np.random.default_rng(self.seed)
        R = self.diameter_m / 2
        nx = int(np.ceil(self.diameter_m / h))
        nz = int(np.ceil(self.thickness_m / h))
        seeds, weights, n_seed = self.calibrate(rng)
        x = (np.arange(nx) - (nx - 1) / 2) * h
        z = (np.arange(nz) - (nz - 1) / 2) * h
        raw = _label_xyz(x, z, R, seeds, weights, pick_labeller(use_gpu, labeller))
        inside = raw >= 0
        keep = np.unique(raw[inside])
        remap = np.full(len(seeds), -1, np.int32)
        remap[keep] = np.arange(len(keep))
        labels = np.full(raw.shape, -1, np.int16)
        labels[inside] = remap[raw[inside]].astype(np.int16)
        axes = sample_watson(len(keep), self.fabric_axis, self.concentration, rng)
        adj = adjacency(labels)
        if self.spatial_corr > 0:
            target_a1 = orientation_tensor(axes)[0][0]
            for _ in range(3):
                nb = np.zeros_like(axes)
                for g, ns in adj.items():
                    if ns:
                        v = axes[list(ns)]
                        v = v * np.sign(v @ axes[g])[:, None]
                        nb[g] = v.mean(axis=0)
                    else:
                        nb[g] = axes[g]
                axes = (1 - self.spatial_corr) * axes + self.spatial_corr * nb
                axes /= np.linalg.norm(axes, axis=1, keepdims=True)
            axes = renormalise_fabric(axes, target_a1)
        return dict(labels=labels, axes=axes, seeds=seeds[keep], weights=weights[keep],
                    adjacency=adj, h=h, inside=inside, shape=labels.shape, n_seed=n_seed)


def pick_labeller(use_gpu=None, labeller=None):
    if labeller is not None:
        if labeller not in ("gpu", "exact", "shortlist"):
            raise ValueError(f"labeller must be 'gpu', 'exact' or 'shortlist', got {labeller!r}")
        return labeller
    if use_gpu is None:
        try:
            import torch
            use_gpu = torch.cuda.is_available()
        except Exception:
            use_gpu = False
    return "gpu" if use_gpu else "shortlist"


def _label_xyz(x, z, R, seeds, weights, how):
    """(nx, nx, nz) int32 power-diagram labels of the cylinder r <= R on the
    square grid x by x by z; -1 outside."""
    if how == "gpu":
        return label_cylinder(x, x, z, R, seeds, weights).cpu().numpy().transpose(2, 1, 0)
    if how == "exact":
        return label_cylinder_numpy(x, x, z, R, seeds, weights).transpose(2, 1, 0)
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    inside = (X ** 2 + Y ** 2) <= R ** 2
    raw = np.full(X.shape, -1, np.int32)
    raw[inside] = assign_shortlist(np.stack([X[inside], Y[inside], Z[inside]], 1), seeds,
                                   weights).astype(np.int32)
    return raw


def rotated_grid_single_raster(build, h, sponge, rot_deg, use_gpu=None, labeller=None):
    """Solver grid of the specimen rotated by -rot_deg about z, labelled by
    evaluating the Laguerre tessellation at the solver points (seeds rotated
    instead of the points; the reference's single_raster path,
    sim/core/rotation_test.py:93-127). Returns (lab, nd, m, axes_rot)."""
    labels, h_spec = build["labels"], build["h"]
    nx_s, _, nz_s = labels.shape
    D = nx_s * h_spec
    nd = int(round(D / h))
    ndz = int(round(nz_s * h_spec / h))
    a = np.radians(rot_deg)
    ca, sa = np.cos(a), np.sin(a)
    u = (np.arange(nd) + 0.5) * h - D / 2.0
    Rd = 0.5 * D
    zc = (np.arange(ndz) - (ndz - 1) / 2) * h
    Rm = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])
    sd = np.asarray(build["seeds"], float) @ Rm
    wts = np.asarray(build["weights"], float)
    core = _label_xyz(u, zc, Rd, sd, wts, pick_labeller(use_gpu, labeller)).transpose(2, 1, 0)
    m = sponge + 3
    nz, nx = ndz + 2 * m, nd + 2 * m
    lab = np.full((nz, nx, nx), -1, np.int32)
    lab[m:m + ndz, m:m + nd, m:m + nd] = core
    return lab, nd, m, np.asarray(build["axes"], float) @ Rm


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


def rotated_grid_device(labels_xyz, axes, h_spec, h, sponge, rot_deg, device=None):
    """rotated_grid on the GPU (pe_rotated_grid): the same (lab, nd, m,
    axes_rot), bit for bit, with lab a device int32 tensor. labels_xyz: the
    specimen labels (x, y, z), numpy or a device tensor."""
    from . import _capi
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("rotated_grid_device runs on a CUDA device; use rotated_grid on CPU")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if isinstance(labels_xyz, torch.Tensor):
        lab_in = labels_xyz.to(device=dev, dtype=torch.int32).contiguous()
    else:
        lab_in = torch.from_numpy(np.ascontiguousarray(labels_xyz, np.int32)).to(dev)
    nx_s, _, nz_s = lab_in.shape
    D = nx_s * h_spec
    nd = int(round(D / h))
    ndz = int(round(nz_s * h_spec / h))
    a = np.radians(rot_deg)
    ca, sa = np.cos(a), np.sin(a)
    m = sponge + 3
    out = torch.empty((ndz + 2 * m, nd + 2 * m, nd + 2 * m), dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        _capi.check(_capi.lib().pe_rotated_grid(
            lab_in.data_ptr(), nx_s, nz_s, float(h_spec), float(h), nd, ndz, float(ca), float(sa), m,
            out.data_ptr(), _capi.C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    R = np.array([[ca, -sa, 0.0], [sa, ca, 0.0], [0.0, 0.0, 1.0]])
    return out, nd, m, np.asarray(axes, float) @ R


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
