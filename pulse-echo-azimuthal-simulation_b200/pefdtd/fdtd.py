"""Drop-in replacement for the reference solver module ``sim/core/fdtd.py``.

Same entry points, argument meaning and error behaviour as the reference
(Jerome-Graves/pulse-echo-azimuthal-simulation):

  forward_fused_labels  sim/core/fdtd.py:1618-1816  (production label path)
  forward_fused         sim/core/fdtd.py:831-921    (dense per-cell stiffness)
  forward               sim/core/fdtd.py:236-376    (array path)
  material_tables, safe_dt_labels, optimised_coeffs, taylor_coeffs,
  cfl_limit, sponge_profile, face_density, max_grid_speed, safe_dt, ricker,
  pick_peak, detrend_hp, absorption_mask  (re-exported host helpers)

Every solve runs on the GPU through the C ABI of include/pefdtd.h; there is
no CPU path. Device memory is PyTorch-owned (the nine state fields and the
trace buffer); the solver copies labels, tables and probe lists into its own
buffers.

Extensions over the reference, all keyword-only and off by default:
  dtype="float64"        run the same kernels in FP64 (the reference's label
                         path is FP32 only; its array path on CPU is FP64)
  damped_record=True     record pressure from the end-of-step damped stress,
                         the convention of forward_fused / forward; this
                         lifts the reference's refusal of source/receiver cells
                         inside the sponge (:1705-1722), which exists only
                         because its label path records pre-damp stress
  device=                torch device (default: current CUDA device)
  chunk_steps / tile / z_chunk   launch schedule (see pefdtd.autotune)
Labels may reach PE_MAX_MATERIALS - 2 (16381) instead of the reference's
uint8 limit of 254; the device label volume is uint16.
"""
from __future__ import annotations

import numpy as np

from . import _capi
from .coeffs import cfl_limit, optimised_coeffs, ppw_for_error, taylor_coeffs  # noqa: F401
from .damping import (absorption_mask, face_density, max_grid_speed, safe_dt,  # noqa: F401
                      safe_dt_labels, sponge_axis_profiles, sponge_profile)
from .materials import c36_to_c21, grain_stiffness, material_tables  # noqa: F401
from .wavelets import detrend_hp, hann_tone_burst, pick_peak, ricker  # noqa: F401

MAX_LABEL = _capi.MAX_MATERIALS - 2

_DT = {"float32": (np.float32, _capi.PE_F32), "float64": (np.float64, _capi.PE_F64)}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pefdtd runs on a CUDA device only; none is available")
    return torch


def _dtype(dtype):
    key = np.dtype(dtype).name
    if key not in _DT:
        raise ValueError(f"dtype must be float32 or float64, got {dtype}")
    return _DT[key]


def _flat_probe(shape, src_pts, rec_groups, npdt):
    """Flat C-order indices and weights (np.ravel_multi_index, :1700-1704)."""
    s_idx = np.array([np.ravel_multi_index(tuple(int(v) for v in i), shape) for i, _ in src_pts],
                     np.int64).reshape(-1)
    s_w = np.array([w for _, w in src_pts], npdt).reshape(-1)
    offs, idx, wts = [0], [], []
    for pts, w in rec_groups:
        q = np.array([np.ravel_multi_index(tuple(int(v) for v in p), shape) for p in pts],
                     np.int64).reshape(-1)
        idx.append(q)
        wts.append(np.asarray(w, npdt).reshape(-1))
        if len(wts[-1]) != len(q):
            raise ValueError("receiver group weights and points differ in length")
        offs.append(offs[-1] + len(q))
    r_idx = np.concatenate(idx) if idx else np.zeros(0, np.int64)
    r_w = np.concatenate(wts) if wts else np.zeros(0, npdt)
    return s_idx, s_w, np.array(offs, np.int64), r_idx, r_w


def c_solve_structs(mats, Ct, rho_t, h, dt, coeffs, src_idx, src_w, rec_off, rec_idx, rec_w,
                    record="pressure", damped_record=False, sponge=None, damp_volume=None,
                    dtype="float32", device=None, chunk_steps=0, tile=(0, 0), z_chunk=0,
                    variant="tiled"):
    """The C ABI description of one solve (PeConfig, PeMedium, PeProbe) plus
    the host arrays and device tensors it points at, which must stay alive
    until the solver has been created."""
    torch = _torch()
    npdt, pedt = _dtype(dtype)
    on_device = isinstance(mats, torch.Tensor)   # material indices already on the device
    if not on_device:
        mats = np.asarray(mats)
    shape = tuple(int(v) for v in mats.shape)
    nz, ny, nx = shape
    coeffs = np.asarray(coeffs, float).reshape(-1)
    if record not in _capi.REC_KIND:
        raise ValueError(f"record must be one of {sorted(_capi.REC_KIND)}, got {record!r}")
    if variant not in _capi.KERNEL_VARIANT:
        raise ValueError(f"variant must be one of {sorted(_capi.KERNEL_VARIANT)}")
    cfg = _capi.PeConfig()
    cfg.nz, cfg.ny, cfg.nx = nz, ny, nx
    cfg.dtype = pedt
    cfg.n_coeffs = len(coeffs)
    for j, c in enumerate(coeffs[:4]):
        cfg.coeffs[j] = float(c)
    cfg.h, cfg.dt = float(h), float(dt)
    cfg.record = _capi.REC_KIND[record]
    cfg.damped_record = int(bool(damped_record))
    Ct = np.ascontiguousarray(np.asarray(Ct, npdt).reshape(-1, 36))
    rho_t = np.ascontiguousarray(np.asarray(rho_t, npdt).reshape(-1))
    cfg.n_mat = len(rho_t)
    cfg.chunk_steps = int(chunk_steps)
    cfg.tile_x, cfg.tile_y = int(tile[0]), int(tile[1])
    cfg.z_chunk = int(z_chunk)
    cfg.variant = _capi.KERNEL_VARIANT[variant]
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    with torch.cuda.device(dev):
        if on_device:
            # indices below 2^14 (the flag bits are set by the solver): int16 holds them
            lab_t = mats.to(device=dev, dtype=torch.int16).contiguous()
        else:
            lab_t = torch.from_numpy(np.ascontiguousarray(mats.astype(np.uint16).view(np.int16))).to(dev)
        dvol_t = (torch.from_numpy(np.ascontiguousarray(damp_volume, np.float32)).to(dev)
                  if damp_volume is not None else None)
    keep = [lab_t, dvol_t, Ct, rho_t]
    md = _capi.PeMedium()
    md.labels_dev = lab_t.data_ptr()
    md.damp_volume_dev = dvol_t.data_ptr() if dvol_t is not None else None
    md.ctab, md.rho = _capi.ptr(Ct), _capi.ptr(rho_t)
    if sponge is not None:
        sp = [np.ascontiguousarray(p, np.float32) for p in sponge]
        keep += sp
        md.sponge_z, md.sponge_y, md.sponge_x = [_capi.ptr(p) for p in sp]
    pr = _capi.PeProbe()
    src_idx = np.ascontiguousarray(src_idx, np.int64)
    src_w = np.ascontiguousarray(src_w, npdt)
    rec_off = np.ascontiguousarray(rec_off, np.int64)
    rec_idx = np.ascontiguousarray(rec_idx, np.int64)
    rec_w = np.ascontiguousarray(rec_w, npdt)
    keep += [src_idx, src_w, rec_off, rec_idx, rec_w]
    pr.n_src = len(src_idx)
    pr.src_idx, pr.src_w = _capi.ptr(src_idx), _capi.ptr(src_w)
    pr.n_groups = len(rec_off) - 1
    pr.rec_off, pr.rec_idx, pr.rec_w = _capi.ptr(rec_off), _capi.ptr(rec_idx), _capi.ptr(rec_w)
    return dict(cfg=cfg, md=md, pr=pr, keep=keep, shape=shape, n_groups=len(rec_off) - 1)


class DeviceSolve:
    """One solve held on the GPU: state, solver handle and trace buffer.

    mats: (nz, ny, nx) material indices (label + 1), any integer array.
    Ct: (n_mat, 36) stiffness rows, rho_t: (n_mat,) densities.
    """

    def __init__(self, mats, Ct, rho_t, h, dt, coeffs, src_idx, src_w, rec_off, rec_idx, rec_w,
                 record="pressure", damped_record=False, sponge=None, damp_volume=None,
                 dtype="float32", device=None, chunk_steps=0, tile=(0, 0), z_chunk=0,
                 variant="tiled"):
        torch = _torch()
        npdt, pedt = _dtype(dtype)
        self.torch = torch
        self.npdt = npdt
        self.tdt = torch.float64 if npdt == np.float64 else torch.float32
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        S = c_solve_structs(mats, Ct, rho_t, h, dt, coeffs, src_idx, src_w, rec_off, rec_idx, rec_w,
                            record, damped_record, sponge, damp_volume, dtype, self.device,
                            chunk_steps, tile, z_chunk, variant)
        cfg, md, pr, keep = S["cfg"], S["md"], S["pr"], S["keep"]
        self.shape = S["shape"]
        nz, ny, nx = self.shape
        self.n_groups = S["n_groups"]
        self.cfg = cfg
        with torch.cuda.device(self.device):
            self.state = torch.zeros((9, nz, ny, nx), dtype=self.tdt, device=self.device)
        L = _capi.lib()
        h_ = _capi.C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.check(L.pe_solver_create(_capi.C.byref(cfg), _capi.C.byref(md), _capi.C.byref(pr),
                                           _capi.C.byref(h_)))
        self._h = h_
        self._L = L
        st = _capi.PeState()
        for i in range(3):
            st.v[i] = self.state[i].data_ptr()
        for i in range(6):
            st.s[i] = self.state[3 + i].data_ptr()
        self._st = st
        self.traces = None
        self.nt = 0
        del keep

    def set_wavelet(self, wavelet):
        w = np.ascontiguousarray(np.asarray(wavelet, float).astype(self.npdt).reshape(-1))
        _capi.check(self._L.pe_solver_set_wavelet(self._h, _capi.ptr(w), len(w)))
        self.nt = len(w)
        with self.torch.cuda.device(self.device):
            self.traces = self.torch.zeros((max(self.nt, 1), max(self.n_groups, 1)),
                                           dtype=self.tdt, device=self.device)

    def reset(self):
        self.state.zero_()

    def run(self, n0, n1, stream=None):
        torch = self.torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _capi.check(self._L.pe_solver_run(self._h, _capi.C.byref(self._st),
                                              self.traces.data_ptr(), int(n0), int(n1),
                                              _capi.C.c_void_p(stream.cuda_stream)))

    def launch_count(self):
        return int(self._L.pe_solver_launch_count(self._h))

    def profile(self, n_steps, stream=None):
        """Mean per-step (stress_ms, velocity_ms) over n_steps from step 0;
        advances the state."""
        torch = self.torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        ms = (_capi.C.c_float * 2)()
        with torch.cuda.device(self.device):
            _capi.check(self._L.pe_solver_profile(self._h, _capi.C.byref(self._st), int(n_steps),
                                                  ms, _capi.C.c_void_p(stream.cuda_stream)))
        return float(ms[0]), float(ms[1])

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.pe_solver_destroy(self._h)
            self._h = _capi.C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check_status(self):
        """Raise if a bounded device-side wait of the queued work gave up."""
        _capi.check(self._L.pe_solver_status(self._h))

    def traces_numpy(self, nt=None):
        nt = self.nt if nt is None else nt
        self.check_status()
        return self.traces[:nt, :self.n_groups].cpu().numpy()


def _run_with_progress(solve, nt, progress):
    """Queue the steps; call progress(n / nt) after every step n with
    n % 200 == 0, as the reference does (:1814-1815). An exception from the
    callback abandons the solve."""
    if progress is None:
        solve.run(0, nt)
        return
    n = 0
    while n < nt:
        nxt = min(nt, n + 1 if n % 200 == 0 else (n // 200 + 1) * 200 + 1)
        solve.run(n, nxt)
        last = nxt - 1
        if last % 200 == 0:
            progress(last / nt)
        n = nxt


def _coeffs_or_default(coeffs, order):
    if coeffs is None:
        coeffs = optimised_coeffs(order)
    return np.asarray(coeffs, float).reshape(-1)


def label_solve_spec(lab, axes, h, dt, nt, src_pts, wavelet, rec_groups, order=8, coeffs=None,
                     sponge_width=0, sponge_strength=0.09, damp_mask=None, c_couplant=1500.0,
                     rho_couplant=300.0, record="pressure", mat_tables=None, *, dtype="float32",
                     damped_record=False):
    """Host half of :func:`forward_fused_labels`: checks its arguments as the
    reference does (:1638-1722) and returns the solve description
    (keyword arguments of :func:`c_solve_structs` plus ``wavelet``) that
    :class:`DeviceSolve` and :class:`pefdtd.batch.BatchSolver` take."""
    coeffs = _coeffs_or_default(coeffs, order)
    if len(coeffs) > 4:
        raise ValueError(
            f"forward_fused_labels supports order <= 8 ({len(coeffs)} coefficients given): "
            f"the kernels carry +/-4 taps per axis.")
    lab = np.asarray(lab)
    if lab.ndim != 3:
        raise ValueError("lab must be a (nz, ny, nx) volume")
    lmin, lmax = int(lab.min()), int(lab.max())
    if lmin < -1 or lmax > MAX_LABEL:
        raise ValueError(f"labels must lie in [-1, {MAX_LABEL}]; got [{lmin}, {lmax}]")
    npdt, _ = _dtype(dtype)
    if mat_tables is None:
        if lmax >= len(axes):
            raise ValueError(f"label {lmax} has no c-axis (len(axes) = {len(axes)}).")
        if npdt == np.float64:
            Ct, rho_t = _material_tables64(axes, c_couplant, rho_couplant)
        else:
            Ct, rho_t = material_tables(axes, c_couplant, rho_couplant)
    else:
        Ct, rho_t = mat_tables
        rho_t = np.ascontiguousarray(rho_t, np.float32 if npdt == np.float32 else np.float64)
        Ct = np.ascontiguousarray(Ct, rho_t.dtype).reshape(len(rho_t), 36)
        if lmax + 1 >= len(rho_t):
            raise ValueError(f"label {lmax} has no row in mat_tables "
                             f"(n_mat = {len(rho_t)}, need >= {lmax + 2}).")
    shape = lab.shape
    mats = (lab + 1).astype(np.uint16)
    sponge = sponge_axis_profiles(shape, sponge_width, sponge_strength) if sponge_width > 0 else None
    dm = np.ascontiguousarray(damp_mask, np.float32) if damp_mask is not None else None
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, src_pts, rec_groups, npdt)
    if not damped_record and (sponge is not None or dm is not None):
        cells = np.concatenate([s_idx, r_idx])
        if len(cells):
            d = _damp_at(cells, shape, sponge, dm)
            bad = cells[d < 0.999]
            if len(bad):
                raise ValueError(
                    f"{len(bad)} source/receiver cells sit where damp < 0.999 (e.g. flat index "
                    f"{int(bad[0])}): the deferred-damping scheme records pre-damp stress there "
                    f"and would silently diverge from the dense path. Move the footprint out of "
                    f"the sponge/fluid-damped region (or pass damped_record=True).")
    return dict(mats=mats, Ct=Ct, rho_t=rho_t, h=h, dt=dt, coeffs=coeffs, src_idx=s_idx,
                src_w=s_w, rec_off=r_off, rec_idx=r_idx, rec_w=r_w, record=record,
                damped_record=damped_record, sponge=sponge, damp_volume=dm,
                wavelet=np.asarray(wavelet, float)[:int(nt)])


def forward_fused_labels(lab, axes, h, dt, nt, src_pts, wavelet, rec_groups, order=8,
                         coeffs=None, sponge_width=0, sponge_strength=0.09, damp_mask=None,
                         c_couplant=1500.0, rho_couplant=300.0, record="pressure", slab=32,
                         stress_smem=False, progress=None, mat_tables=None, *,
                         dtype="float32", damped_record=False, device=None, chunk_steps=0,
                         tile=(0, 0), z_chunk=0, variant="tiled", return_solve=False):
    """Label-indexed solve; returns the (nt, n_rec) traces as float32 (float64
    when dtype="float64"). ``slab`` and ``stress_smem`` are accepted for
    signature compatibility; the kernels march z without slabs."""
    sp = label_solve_spec(lab, axes, h, dt, nt, src_pts, wavelet, rec_groups, order, coeffs,
                          sponge_width, sponge_strength, damp_mask, c_couplant, rho_couplant,
                          record, mat_tables, dtype=dtype, damped_record=damped_record)
    wav = sp.pop("wavelet")
    solve = DeviceSolve(sp.pop("mats"), sp.pop("Ct"), sp.pop("rho_t"), sp.pop("h"), sp.pop("dt"),
                        sp.pop("coeffs"), sp.pop("src_idx"), sp.pop("src_w"), sp.pop("rec_off"),
                        sp.pop("rec_idx"), sp.pop("rec_w"), **sp, dtype=dtype, device=device,
                        chunk_steps=chunk_steps, tile=tile, z_chunk=z_chunk, variant=variant)
    solve.set_wavelet(wav)
    try:
        _run_with_progress(solve, int(nt), progress)
        out = solve.traces_numpy(int(nt))
    finally:
        if not return_solve:
            solve.close()
    return (out, solve) if return_solve else out


def _material_tables64(axes, c_couplant, rho_couplant):
    """FP64 tables: the same construction without the final f32 rounding."""
    axes = np.asarray(axes, float).reshape(-1, 3)
    n_mat = len(axes) + 1
    C = np.zeros((n_mat, 6, 6))
    C[0, :3, :3] = rho_couplant * c_couplant * c_couplant
    if len(axes):
        C[1:] = grain_stiffness(axes)
    iu = np.triu_indices(6)
    C[:, iu[1], iu[0]] = C[:, iu[0], iu[1]]
    rho = np.full(n_mat, 917.0)
    rho[0] = rho_couplant
    return C.reshape(n_mat, 36), rho


def _damp_at(cells, shape, sponge, dm):
    iz, iy, ix = np.unravel_index(cells, shape)
    d = np.ones(len(cells), np.float32)
    if sponge is not None:
        d = (sponge[0][iz] * sponge[1][iy]) * sponge[2][ix]
    if dm is not None:
        d = d * dm.reshape(-1)[cells] if sponge is not None else dm.reshape(-1)[cells]
    return d


def _media_rows(C, rho):
    """Per-cell stiffness dict + density -> (ncell, 22) rows [C21..., rho]."""
    rho = np.asarray(rho, float)
    shape = rho.shape
    keys = [f"C{i + 1}{j + 1}" for i in range(6) for j in range(i, 6)]
    cols = []
    for k in keys:
        a = np.asarray(C.get(k, 0.0), float)
        cols.append(np.broadcast_to(a, shape).reshape(-1))
    cols.append(rho.reshape(-1))
    return np.stack(cols, axis=1), shape


def _rows_to_tables(rows, npdt):
    C21 = rows[:, :21]
    Ct = np.zeros((len(rows), 6, 6))
    for k, (i, j) in enumerate([(i, j) for i in range(6) for j in range(i, 6)]):
        Ct[:, i, j] = C21[:, k]
        Ct[:, j, i] = C21[:, k]
    return Ct.reshape(-1, 36).astype(npdt), rows[:, 21].astype(npdt)


def _compress_dense(C, rho, npdt, media="auto"):
    """Per-cell stiffness dict + density -> (mats, Ct, rho_t, variant).

    media="table": one table row per distinct (C21, rho) combination (the
    label kernels; at most MAX_MATERIALS rows); "dense": one row per cell
    (the per-cell kernel variant, any medium, the reference's dense path);
    "auto": the table when the distinct media fit it, else per cell."""
    if media not in ("auto", "table", "dense"):
        raise ValueError(f"media must be auto, table or dense, got {media!r}")
    M, shape = _media_rows(C, rho)
    if media != "dense":
        rows, inv = np.unique(M, axis=0, return_inverse=True)
        if len(rows) <= _capi.MAX_MATERIALS:
            Ct, rho_t = _rows_to_tables(rows, npdt)
            return inv.reshape(shape).astype(np.uint16), Ct, rho_t, None
        if media == "table":
            raise ValueError(f"{len(rows)} distinct media exceed the {_capi.MAX_MATERIALS}-row table")
    Ct, rho_t = _rows_to_tables(M, npdt)
    return np.zeros(shape, np.uint16), Ct, rho_t, "dense"


def forward_fused(C, rho, h, dt, nt, src_pts, wavelet, rec_groups, order=8, coeffs=None,
                  sponge_width=0, sponge_strength=0.09, damp_mask=None, record="pressure",
                  progress=None, *, dtype="float32", device=None, chunk_steps=0, tile=(0, 0),
                  z_chunk=0, variant="tiled", media="auto"):
    """Dense-stiffness solve (C: dict of the 21 Voigt maps or scalars, rho:
    (nz, ny, nx)), with the dense path's end-of-step damped recording.
    Distinct media are folded into a material table and run on the label
    kernels when they fit it (at most MAX_MATERIALS); otherwise (or with
    media="dense") every cell keeps its own row and the per-cell kernel
    variant runs (the reference's K1-K3 take any per-cell medium,
    sim/core/fdtd.py:392-583)."""
    coeffs = _coeffs_or_default(coeffs, order)
    if len(coeffs) > 4:
        raise ValueError(f"order <= 8 supported ({len(coeffs)} coefficients given)")
    npdt, _ = _dtype(dtype)
    mats, Ct, rho_t, forced = _compress_dense(C, rho, npdt, media)
    if forced is not None:
        variant = forced
    shape = mats.shape
    sponge = sponge_axis_profiles(shape, sponge_width, sponge_strength) if sponge_width > 0 else None
    dm = np.ascontiguousarray(damp_mask, np.float32) if damp_mask is not None else None
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, src_pts, rec_groups, npdt)
    solve = DeviceSolve(mats, Ct, rho_t, h, dt, coeffs, s_idx, s_w, r_off, r_idx, r_w,
                        record=record, damped_record=True, sponge=sponge, damp_volume=dm,
                        dtype=dtype, device=device, chunk_steps=chunk_steps, tile=tile,
                        z_chunk=z_chunk, variant=variant)
    try:
        solve.set_wavelet(np.asarray(wavelet, float)[:nt])
        _run_with_progress(solve, int(nt), progress)
        return solve.traces_numpy(int(nt))
    finally:
        solve.close()


def forward(C, rho, h, dt, nt, src_pts, wavelet, rec_groups, order=8, coeffs=None,
            sponge_width=0, sponge_strength=0.09, device="auto", record="pressure",
            progress=None, *, media="auto"):
    """Array-path signature (:236-238). The reference computes in FP64 on the
    CPU and FP32 on a GPU; here device="cpu" selects the FP64 kernels and
    anything else FP32, both on the GPU. Repeated source cells add their
    weights, as the array path's per-point loop does (:344-346)."""
    if device not in ("auto", "gpu", "cpu"):
        raise ValueError(f"device must be auto, gpu or cpu, got {device!r}")
    dtype = "float64" if device == "cpu" else "float32"
    merged = {}
    for idx, w in src_pts:
        key = tuple(int(v) for v in idx)
        merged[key] = merged.get(key, 0.0) + float(w)
    src = [(k, w) for k, w in merged.items()]
    out = forward_fused(C, rho, h, dt, nt, src, wavelet, rec_groups, order=order, coeffs=coeffs,
                        sponge_width=sponge_width, sponge_strength=sponge_strength,
                        record=record, progress=progress, dtype=dtype, media=media)
    return out.astype(np.float64)
