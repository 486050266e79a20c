"""Gradients of trace misfits through the FDTD solver (hand-written adjoint).

The reference's only FDTD gradient is ringfwi's order-2, undamped,
cell-density adjoint that stores the whole velocity history
(vendor/ringfwi/elastic3d.py:276-463), chained to per-voxel c-axis angles by
vendor/ringfwi/axisfield.py:37-161. Here:

* :class:`AdjointSolve` runs the production forward scheme on the GPU,
  keeping full-state checkpoints every ``checkpoint_every`` steps (in device
  memory, or in pinned host memory with ``offload=True``); the reverse sweep
  recomputes each segment from its checkpoint and applies the exact discrete
  adjoint step (csrc/pe_adjoint.cuh) backwards through it, accumulating
  dJ/dC for every material's 21 stiffness constants. With ``inner_every=m``
  the checkpointing is two-level: a segment is first recomputed keeping
  full-state checkpoints every m steps, and only m steps of velocity history
  are held at a time (memory ~ (K/m) states + m velocity fields instead of
  K velocity fields; ``plan_memory`` picks K, m and the offload for a byte
  budget). The reference keeps the whole velocity history
  (vendor/ringfwi/elastic3d.py:301,305).
* :class:`StiffnessTraces` is a ``torch.autograd.Function`` from the
  per-material table ``(n_mat, 21)`` to the traces ``(nt, n_groups)``; its
  backward is that adjoint with the incoming trace gradient as the adjoint
  source, so any loss on the traces (``0.5*||tr - d||^2`` gives the
  reference's misfit) differentiates through it.
* :func:`misfit_gradients` runs the misfits and gradients of many solves
  together, their segments interleaved on one CUDA stream per solve, in
  waves whose device memory fits the free HBM.
* :func:`ice_table21` builds that table differentiably from per-grain c-axis
  angles (colatitude theta, azimuth phi; R = Rz(phi) Ry(theta), the
  convention of vendor/ringfwi/axisfield.py:37-65 and cof.axes_from_params),
  and :func:`fabric_axes` maps 3 fabric parameters to per-grain axes, so
  gradients reach grain angles and fabric parameters through torch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .fdtd import DeviceSolve, _torch
from .materials import C21_INDEX, ICE, ti_stiffness_6


class _PeAdjoint(C.Structure):
    _fields_ = [("lv", C.c_void_p * 3), ("ls", C.c_void_p * 6), ("v_prev", C.c_void_p * 3),
                ("scratch", C.c_void_p), ("grad", C.c_void_p)]


def _bind():
    L = _capi.lib()
    if not getattr(L, "_adj_bound", False):
        L.pe_solver_adjoint_step.argtypes = [C.c_void_p, C.POINTER(_PeAdjoint), C.c_int64, C.c_void_p,
                                             C.c_void_p]
        L.pe_solver_adjoint_segment.argtypes = [C.c_void_p, C.POINTER(_capi.PeState), C.POINTER(_PeAdjoint),
                                                C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L._adj_bound = True
    return L


def adjoint_bytes(shape, nt, checkpoint_every=200, inner_every=None, offload=False, esize=4,
                  damp_volume=False):
    """Device bytes of one misfit-and-gradient solve (AdjointSolve): the
    solver (state, labels, damping volume), the outer checkpoints (none on
    the device when offloaded), the inner checkpoints and velocity history of
    one reverse segment, and the adjoint state with its 33-field scratch."""
    ncell = int(np.prod(shape))
    field = ncell * esize
    K = max(1, int(checkpoint_every))
    m = min(K, int(inner_every)) if inner_every else K
    solve = 9 * field + 2 * ncell + (4 * ncell if damp_volume else 0)
    outer = 0 if offload else -(-int(nt) // K) * 9 * field
    inner = (-(-min(K, int(nt)) // m)) * 9 * field if m < K else 0
    hist = min(m, int(nt)) * 3 * field
    adj = (9 + 33) * field
    return solve + outer + inner + hist + adj


def plan_memory(shape, nt, budget_bytes, checkpoint_every=200, esize=4, damp_volume=False):
    """(inner_every, offload) for one solve under budget_bytes of device
    memory, preferring no recomputation, then two-level checkpointing with
    the inner spacing that minimises memory (m ~ sqrt(3 K): K/m states of 9
    fields against m velocity fields of 3), then offloading the outer
    checkpoints to pinned host memory. None if even that does not fit."""
    K = max(1, int(checkpoint_every))
    m_best = max(1, min(K, int(round(np.sqrt(3.0 * K)))))
    for inner, off in ((None, False), (m_best, False), (None, True), (m_best, True)):
        if adjoint_bytes(shape, nt, K, inner, off, esize, damp_volume) <= budget_bytes:
            return inner, off
    return None


class AdjointSolve:
    """Forward with checkpoints, then reverse sweeps, on one DeviceSolve."""

    def __init__(self, solve: DeviceSolve, checkpoint_every=200, inner_every=None, offload=False):
        self.solve = solve
        self.K = int(checkpoint_every)
        if self.K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.m = self.K if not inner_every else min(self.K, int(inner_every))
        if self.m < 1:
            raise ValueError("inner_every must be >= 1")
        self.offload = bool(offload)
        self.torch = solve.torch
        self.ckpt = {}
        self.nt = 0

    def _save(self, state):
        if self.offload:
            h = self.torch.empty(state.shape, dtype=state.dtype, device="cpu", pin_memory=True)
            h.copy_(state, non_blocking=True)   # stream-ordered before the next steps
            return h
        return state.clone()

    def forward(self, nt=None):
        """Traces (nt, n_groups) as a device tensor; keeps checkpoints."""
        for _ in self.forward_segments(nt):
            pass
        self.solve.check_status()
        return self.solve.traces[:self.nt, :self.solve.n_groups]

    def forward_segments(self, nt=None):
        """Generator form of :meth:`forward`: each iteration issues one
        checkpoint segment on the current stream, without synchronising."""
        s = self.solve
        nt = s.nt if nt is None else int(nt)
        s.reset()
        self.ckpt = {}
        self.nt = nt
        for a in range(0, nt, self.K):
            self.ckpt[a] = self._save(s.state)
            s.run(a, min(a + self.K, nt))
            yield a

    def backward(self, residual):
        """dJ/dC (n_mat, 21) float64 for the trace adjoint `residual`
        (nt, n_groups): for J = 0.5 ||traces - d||^2 it is traces - d."""
        grad = None
        for grad in self.backward_segments(residual):
            pass
        self.solve.check_status()
        return grad.cpu().numpy()

    def backward_segments(self, residual):
        """Generator form of :meth:`backward`: allocates the adjoint state,
        then each iteration issues the recompute and reverse sweep of one
        segment (last first) on the current stream and yields the device
        gradient accumulated so far ((n_mat, 21) float64)."""
        torch = self.torch
        s = self.solve
        nt, ng = self.nt, s.n_groups
        dev, tdt = s.device, s.tdt
        shape = s.shape
        if isinstance(residual, torch.Tensor):
            res = residual.to(device=dev, dtype=tdt).reshape(nt, ng).contiguous()
        else:
            res = torch.as_tensor(np.asarray(residual), dtype=tdt).reshape(nt, ng).to(dev).contiguous()
        L = _bind()
        with torch.cuda.device(dev):
            lam = torch.zeros((9,) + shape, dtype=tdt, device=dev)
            scratch = torch.zeros((33,) + shape, dtype=tdt, device=dev)
            grad = torch.zeros((s.cfg.n_mat, 21), dtype=torch.float64, device=dev)
            hist = torch.empty((min(self.m, nt), 3) + shape, dtype=tdt, device=dev)
        adj = _PeAdjoint()
        for i in range(3):
            adj.lv[i] = lam[i].data_ptr()
        for i in range(6):
            adj.ls[i] = lam[3 + i].data_ptr()
        adj.scratch = scratch.data_ptr()
        adj.grad = grad.data_ptr()
        stream = torch.cuda.current_stream(dev)

        def reverse(a, b):
            # recompute [a, b) from the state and step back through it in one C call
            with torch.cuda.device(dev):
                _capi.check(L.pe_solver_adjoint_segment(s._h, C.byref(s._st), C.byref(adj), hist.data_ptr(),
                                                        a, b, res.data_ptr(), C.c_void_p(stream.cuda_stream)))

        for a in reversed(sorted(self.ckpt)):
            b = min(a + self.K, nt)
            s.state.copy_(self.ckpt[a], non_blocking=True)
            if self.m >= b - a:
                reverse(a, b)
            else:
                # two levels: inner checkpoints every m steps of the segment,
                # then the sub-segments last first, m steps of history each
                inner = {}
                for a2 in range(a, b, self.m):
                    inner[a2] = s.state.clone()
                    s.run(a2, min(a2 + self.m, b))
                for a2 in reversed(sorted(inner)):
                    s.state.copy_(inner[a2])
                    reverse(a2, min(a2 + self.m, b))
                del inner
            yield grad


def misfit_gradients(problems, c21s, dobs, memory_budget=None, plan=True):
    """J_i = 0.5 ||traces_i(c21_i) - dobs_i||^2 and dJ_i/dc21_i for many
    problems at once (a sweep's azimuths, an inversion's specimens): the
    checkpoint segments of every solve, forward then reverse, are issued
    round-robin on one CUDA stream per solve, so that solves too small to
    fill the GPU run side by side. Per solve the same kernels run in the same
    order as in the one-at-a-time gradient; only the order of the gradient's
    atomic float64 sums may differ.

    The solves run in waves: each wave holds as many solves as fit
    ``memory_budget`` bytes of device memory (default: 80 % of the free
    memory when the call starts), each solve's checkpointing chosen by
    plan_memory for its share when ``plan`` is set (two-level checkpoints,
    host offload) so that even one large solve fits. Returns a list of
    (J, grad (n_mat_i, 21) float64 numpy)."""
    torch = _torch()
    if not (len(problems) == len(c21s) == len(dobs)):
        raise ValueError("one table and one observed record per problem")
    if not problems:
        return []
    if memory_budget is None:
        dev = problems[0].device
        with torch.cuda.device(dev if dev is not None else torch.cuda.current_device()):
            memory_budget = int(0.8 * torch.cuda.mem_get_info()[0])
    waves = plan_waves(problems, memory_budget, plan=plan)
    out = [None] * len(problems)
    for wave in waves:
        res = _misfit_gradients_wave([problems[i] for i, _ in wave], [c21s[i] for i, _ in wave],
                                     [dobs[i] for i, _ in wave], [opt for _, opt in wave])
        for (i, _), r in zip(wave, res):
            out[i] = r
    return out


def plan_waves(problems, budget, plan=True):
    """Groups of (problem index, (inner_every, offload)) whose summed
    adjoint_bytes fit the budget, in problem order."""
    waves, cur, used = [], [], 0
    for i, p in enumerate(problems):
        shape = p.mats.shape
        nt = len(p.wavelet)
        es = 8 if p.dtype in ("float64", np.float64) else 4
        dv = p.damp_mask is not None
        opt = (p.inner_every, p.offload)
        need = adjoint_bytes(shape, nt, p.K, opt[0], opt[1], es, dv)
        if plan and need > budget:
            got = plan_memory(shape, nt, budget, p.K, es, dv)
            if got is None:
                raise MemoryError(f"one gradient solve of {shape} x {nt} steps needs more than "
                                  f"{budget / 2**30:.1f} GiB of device memory even with two-level "
                                  "checkpoints and host offload")
            opt = got
            need = adjoint_bytes(shape, nt, p.K, opt[0], opt[1], es, dv)
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append((i, opt))
        used += need
    if cur:
        waves.append(cur)
    return waves


def _misfit_gradients_wave(problems, c21s, dobs, opts):
    torch = _torch()
    adjs = []
    try:
        for p, c, (inner, off) in zip(problems, c21s, opts):
            adjs.append(p.make_adjoint(np.asarray(c, float), inner_every=inner, offload=off))
        streams = [torch.cuda.Stream(device=a.solve.device) for a in adjs]
        for st, a in zip(streams, adjs):
            st.wait_stream(torch.cuda.current_stream(a.solve.device))

        def interleave(jobs):
            live = list(jobs)
            while live:
                nxt = []
                for st, g in live:
                    with torch.cuda.stream(st):
                        if next(g, None) is not None:
                            nxt.append((st, g))
                live = nxt

        interleave([(st, a.forward_segments()) for st, a in zip(streams, adjs)])
        res, J = [], []
        for st, a, d in zip(streams, adjs, dobs):
            with torch.cuda.stream(st):
                tr = a.solve.traces[:a.nt, :a.solve.n_groups].to(torch.float64)
                r = tr - torch.as_tensor(np.asarray(d, float), device=tr.device).reshape(tr.shape)
                res.append(r)
                J.append(0.5 * (r * r).sum())
        grads = [None] * len(adjs)

        def reverse(k, a, r):
            for g in a.backward_segments(r):
                grads[k] = g
                yield True

        interleave([(st, reverse(k, a, r)) for k, (st, a, r) in enumerate(zip(streams, adjs, res))])
        out = []
        for st, a, j, g in zip(streams, adjs, J, grads):
            st.synchronize()
            a.solve.check_status()
            out.append((float(j.cpu()), g.cpu().numpy()))
        return out
    finally:
        for a in adjs:
            a.solve.close()


# ---------------------------------------------------------------- autograd
class StiffnessTraces:
    """Namespace for the autograd Function (created lazily so that importing
    this module does not require torch)."""
    _fn = None

    @classmethod
    def fn(cls):
        if cls._fn is None:
            torch = _torch()

            class _F(torch.autograd.Function):
                @staticmethod
                def forward(ctx, c21, problem):
                    adj = problem.make_adjoint(c21.detach().cpu().numpy())
                    tr = adj.forward()
                    ctx.adj = adj
                    return tr.detach().to("cpu", torch.float64)

                @staticmethod
                def backward(ctx, grad_tr):
                    g = ctx.adj.backward(grad_tr.detach().cpu().numpy())
                    ctx.adj.solve.close()
                    return torch.from_numpy(g), None

            cls._fn = _F
        return cls._fn


class Problem:
    """Everything of a solve except the stiffness table: labels, densities,
    probe, wavelet, damping and scheme. ``traces(c21)`` is differentiable in
    ``c21`` (torch tensor (n_mat, 21))."""

    def __init__(self, mats, rho_t, h, dt, coeffs, src_pts, rec_groups, wavelet, record="vz",
                 sponge_width=0, damp_mask=None, damped_record=True, dtype="float64",
                 checkpoint_every=200, device=None, inner_every=None, offload=False):
        from .damping import sponge_axis_profiles
        from .fdtd import _flat_probe
        self.mats = np.asarray(mats)
        self.rho_t = np.asarray(rho_t, float)
        self.h, self.dt = float(h), float(dt)
        self.coeffs = np.asarray(coeffs, float)
        shape = self.mats.shape
        self.probe = _flat_probe(shape, src_pts, rec_groups, np.float64)
        self.wavelet = np.asarray(wavelet, float)
        self.record = record
        self.sponge = sponge_axis_profiles(shape, sponge_width) if sponge_width > 0 else None
        self.damp_mask = damp_mask
        self.damped_record = damped_record
        self.dtype = dtype
        self.K = checkpoint_every
        self.inner_every = inner_every
        self.offload = offload
        self.device = device

    def make_adjoint(self, c21, inner_every=None, offload=None):
        c21 = np.asarray(c21, float).reshape(-1, 21)
        Ct = np.zeros((len(c21), 6, 6))
        for k, (i, j) in enumerate(C21_INDEX):
            Ct[:, i, j] = c21[:, k]
            Ct[:, j, i] = c21[:, k]
        s_idx, s_w, r_off, r_idx, r_w = self.probe
        solve = DeviceSolve(self.mats, Ct.reshape(-1, 36), self.rho_t, self.h, self.dt, self.coeffs,
                            s_idx, s_w, r_off, r_idx, r_w, record=self.record,
                            damped_record=self.damped_record, sponge=self.sponge,
                            damp_volume=self.damp_mask, dtype=self.dtype, device=self.device)
        solve.set_wavelet(self.wavelet)
        return AdjointSolve(solve, self.K,
                            inner_every=self.inner_every if inner_every is None else inner_every,
                            offload=self.offload if offload is None else offload)

    def traces(self, c21):
        return StiffnessTraces.fn().apply(c21, self)

    def traces_numpy(self, c21):
        """Forward traces (nt, n_groups) for the table c21, no checkpoints."""
        c21 = np.asarray(c21, float).reshape(-1, 21)
        Ct = np.zeros((len(c21), 6, 6))
        for k, (i, j) in enumerate(C21_INDEX):
            Ct[:, i, j] = c21[:, k]
            Ct[:, j, i] = c21[:, k]
        s_idx, s_w, r_off, r_idx, r_w = self.probe
        solve = DeviceSolve(self.mats, Ct.reshape(-1, 36), self.rho_t, self.h, self.dt, self.coeffs,
                            s_idx, s_w, r_off, r_idx, r_w, record=self.record,
                            damped_record=self.damped_record, sponge=self.sponge,
                            damp_volume=self.damp_mask, dtype=self.dtype, device=self.device)
        try:
            solve.set_wavelet(self.wavelet)
            nt = len(self.wavelet)
            solve.run(0, nt)
            solve.check_status()
            return np.asarray(solve.traces_numpy(nt), float)
        finally:
            solve.close()


# ---------------------------------------------------------------- tables from angles
def _host_torch():
    """torch for the host-side angle chain (autograd on float64 CPU tensors;
    no device is needed for it, unlike the solver)."""
    import torch
    return torch


def _bond_torch(A, B):
    """Bilinear Bond form for (P,3,3) tensors; _bond_torch(R, R) = M(R)."""
    torch = _host_torch()
    V = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))
    rows = []
    for (i, j) in V:
        cols = []
        for (k, l) in V:
            v = A[:, i, k] * B[:, j, l]
            if k != l:
                v = v + A[:, i, l] * B[:, j, k]
            cols.append(v)
        rows.append(torch.stack(cols, dim=-1))
    return torch.stack(rows, dim=-2)


def rotation_colat_azim(theta, phi):
    """R = Rz(phi) Ry(theta): maps the crystal c-axis z onto
    (sin t cos p, sin t sin p, cos t)."""
    torch = _host_torch()
    ct, st, cp, sp = torch.cos(theta), torch.sin(theta), torch.cos(phi), torch.sin(phi)
    z, o = torch.zeros_like(theta), torch.ones_like(theta)
    Ry = torch.stack([torch.stack([ct, z, st], -1), torch.stack([z, o, z], -1),
                      torch.stack([-st, z, ct], -1)], -2)
    Rz = torch.stack([torch.stack([cp, -sp, z], -1), torch.stack([sp, cp, z], -1),
                      torch.stack([z, z, o], -1)], -2)
    return Rz @ Ry


def ice_table21(theta, phi, c_couplant=1500.0, rho_couplant=300.0, material=None):
    """(n_g + 1, 21) stiffness table (row 0 the fluid couplant) from per-grain
    c-axis angles, differentiable in theta and phi (torch float64)."""
    torch = _host_torch()
    mat = ICE if material is None else material
    theta = torch.as_tensor(theta, dtype=torch.float64)
    phi = torch.as_tensor(phi, dtype=torch.float64)
    R = rotation_colat_azim(theta, phi)
    M = _bond_torch(R, R)
    C0 = torch.as_tensor(ti_stiffness_6(**mat), dtype=torch.float64)
    Cg = M @ C0 @ M.transpose(-1, -2)
    iu = [i for i, _ in C21_INDEX], [j for _, j in C21_INDEX]
    g21 = Cg[:, iu[0], iu[1]]
    K = rho_couplant * c_couplant * c_couplant
    fl = torch.zeros(1, 21, dtype=torch.float64)
    for k, (i, j) in enumerate(C21_INDEX):
        if i < 3 and j < 3:
            fl[0, k] = K
    return torch.cat([fl, g21], dim=0)


def angles_from_axes(axes):
    """(theta, phi) of unit axes (upper hemisphere; c and -c are the same)."""
    a = np.asarray(axes, float).reshape(-1, 3)
    a = np.where(a[:, 2:3] < 0, -a, a)
    theta = np.arccos(np.clip(a[:, 2], -1, 1))
    phi = np.arctan2(a[:, 1], a[:, 0])
    return theta, phi


def fabric_axes(params, base):
    """Per-grain c-axes from 3 fabric parameters (tilt, azimuth, log_conc)
    and fixed per-grain base directions (n, 3): each base direction is
    stretched by exp(log_conc) along z (> 0 clusters the axes about the pole,
    < 0 spreads them toward a girdle), normalised, then the whole fabric is
    tilted by `tilt` about y and turned by `azimuth` about z. Differentiable;
    a construction of this module (the reference's fabric fits use Watson
    (alpha, kappa) on ray-model observables, sim/model/fit_fabric.py:224-274).
    """
    torch = _host_torch()
    p = torch.as_tensor(params, dtype=torch.float64)
    u = torch.as_tensor(base, dtype=torch.float64)
    s = torch.exp(p[2])
    a = torch.stack([u[:, 0], u[:, 1], u[:, 2] * s], -1)
    a = a / torch.linalg.norm(a, dim=-1, keepdim=True)
    R = rotation_colat_azim(p[0].reshape(1), p[1].reshape(1))[0]
    return a @ R.T


def theta_phi_torch(axes):
    torch = _host_torch()
    z = axes[:, 2]
    sgn = torch.where(z < 0, -torch.ones_like(z), torch.ones_like(z))
    a = axes * sgn[:, None]
    theta = torch.acos(torch.clamp(a[:, 2], -1.0, 1.0))
    phi = torch.atan2(a[:, 1], a[:, 0])
    return theta, phi
