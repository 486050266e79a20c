"""Many independent solves advanced together on one GPU.

The reference runs one solve at a time: an azimuth sweep is a Python loop
over ``forward_fused_labels`` calls (sim/pipeline/sweep_runner.py:322-390),
and its only batching precedent stacks CPU transmits on a leading axis
(vendor/ringfwi/elastic3d.py:474-632). Here every solve of a batch (any grid
size, its own medium, probe, wavelet, state and traces) is advanced by one
stress and one velocity launch per step for the whole batch; the step loop
replays as captured CUDA graphs of ``chunk_steps`` steps, and the work layout
(planes per z-march, graph length) comes from :mod:`pefdtd.autotune`.
"""
from __future__ import annotations

import numpy as np

from . import _capi
from .damping import sponge_axis_profiles
from .fdtd import _dtype, _flat_probe, _torch, c_solve_structs


def spec_from_problem(p, damped_record=True, record=None):
    """Solve description (keyword arguments of c_solve_structs plus the
    wavelet) from a workload problem dict (pefdtd.workloads.make_problem)."""
    shape = p["lab"].shape
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], np.float64)
    return dict(mats=p["mats"], Ct=p["Ct"], rho_t=p["rho_t"], h=p["h"], dt=p["dt"],
                coeffs=p["coeffs"], src_idx=s_idx, src_w=s_w, rec_off=r_off, rec_idx=r_idx,
                rec_w=r_w, record=record or p["record"], damped_record=damped_record,
                sponge=sponge_axis_profiles(shape, p["sponge"]) if p["sponge"] > 0 else None,
                damp_volume=p.get("damp_volume"), wavelet=np.asarray(p["wavelet"], float))


class BatchSolver:
    """A batch of solves on one device. ``specs``: list of dicts from
    :func:`spec_from_problem` (or the same keys)."""

    def __init__(self, specs, dtype="float32", device=None, z_chunk=0, chunk_steps=0):
        torch = _torch()
        self.torch = torch
        self.npdt, _ = _dtype(dtype)
        self.tdt = torch.float64 if self.npdt == np.float64 else torch.float32
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        n = len(specs)
        if n < 1:
            raise ValueError("empty batch")
        built = []
        for sp in specs:
            kw = {k: v for k, v in sp.items() if k != "wavelet"}
            built.append(c_solve_structs(**kw, dtype=dtype, device=self.device,
                                         chunk_steps=chunk_steps, z_chunk=0, variant="tiled"))
        cfgs = (_capi.PeConfig * n)(*[b["cfg"] for b in built])
        mds = (_capi.PeMedium * n)(*[b["md"] for b in built])
        prs = (_capi.PeProbe * n)(*[b["pr"] for b in built])
        L = _capi.lib()
        h = _capi.C.c_void_p()
        with torch.cuda.device(self.device):
            _capi.check(L.pe_batch_create(n, cfgs, mds, prs, _capi.C.byref(h)))
        self._h, self._L = h, L
        self.n = n
        self.shapes = [b["shape"] for b in built]
        self.n_groups = [b["n_groups"] for b in built]
        self.cells = [int(np.prod(s)) for s in self.shapes]
        with torch.cuda.device(self.device):
            self.states = [torch.zeros((9,) + s, dtype=self.tdt, device=self.device) for s in self.shapes]
        self._st = (_capi.PeState * n)()
        for i, st in enumerate(self.states):
            for c in range(3):
                self._st[i].v[c] = st[c].data_ptr()
            for c in range(6):
                self._st[i].s[c] = st[3 + c].data_ptr()
        self.z_chunk, self.chunk_steps = 0, int(chunk_steps)
        self.persistent = False
        self.nt = [0] * n
        self.traces = [None] * n
        self._tr = (_capi.C.c_void_p * n)()
        for i, sp in enumerate(specs):
            self.set_wavelet(i, sp["wavelet"])
        if z_chunk:
            self.schedule(z_chunk, chunk_steps)
        del built

    def set_wavelet(self, i, wavelet):
        w = np.ascontiguousarray(np.asarray(wavelet, float).astype(self.npdt).reshape(-1))
        _capi.check(self._L.pe_batch_set_wavelet(self._h, i, _capi.ptr(w), len(w)))
        self.nt[i] = len(w)
        with self.torch.cuda.device(self.device):
            self.traces[i] = self.torch.zeros((max(len(w), 1), max(self.n_groups[i], 1)),
                                              dtype=self.tdt, device=self.device)
        self._tr[i] = self.traces[i].data_ptr()

    def schedule(self, z_chunk=0, chunk_steps=0):
        _capi.check(self._L.pe_batch_schedule(self._h, int(z_chunk), int(chunk_steps)))
        self.z_chunk, self.chunk_steps = int(z_chunk), int(chunk_steps)

    def set_persistent(self, on=True):
        """Persistent mode: one cooperative launch per graph chunk advances
        every batched solve by all the chunk's steps (grid-wide barriers
        between the stress and velocity phases; bit-identical to the
        per-step launches). FP32 pair-column batches only: returns whether
        the mode is on."""
        rc = self._L.pe_batch_set_persistent(self._h, int(bool(on)))
        if rc == _capi.PE_ERR_UNSUPPORTED and on:
            self.persistent = False
            return False
        _capi.check(rc)
        self.persistent = bool(on)
        return self.persistent

    def reset(self):
        for st in self.states:
            st.zero_()

    def run(self, n0, n1, stream=None):
        torch = self.torch
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _capi.check(self._L.pe_batch_run(self._h, self._st, self._tr, int(n0), int(n1),
                                             _capi.C.c_void_p(stream.cuda_stream)))

    def launch_count(self):
        return int(self._L.pe_batch_launch_count(self._h))

    def check_status(self):
        _capi.check(self._L.pe_batch_status(self._h))

    def traces_numpy(self, nt=None):
        self.check_status()
        out = []
        for i in range(self.n):
            k = self.nt[i] if nt is None else nt
            out.append(self.traces[i][:k, :self.n_groups[i]].cpu().numpy())
        return out

    def cell_updates(self, steps):
        return sum(self.cells) * int(steps)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.pe_batch_destroy(self._h)
            self._h = _capi.C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def forward_batch(problems, nt=None, dtype="float32", device=None, autotune=True, progress=None,
                  damped_record=True):
    """Run a list of workload problems as one batch; returns their traces.

    ``progress(frac)`` is called between graph chunks and may raise to stop.
    """
    from . import autotune as at
    specs = [spec_from_problem(p, damped_record=damped_record) for p in problems]
    nt = min(len(s["wavelet"]) for s in specs) if nt is None else int(nt)
    b = BatchSolver(specs, dtype=dtype, device=device)
    try:
        if autotune:
            at.tune_batch(b)
        step = b.chunk_steps if b.chunk_steps > 0 else 200
        n = 0
        while n < nt:
            m = min(nt, n + step)
            b.run(n, m)
            n = m
            if progress is not None:
                progress(n / nt)
        return b.traces_numpy(nt)
    finally:
        b.close()
