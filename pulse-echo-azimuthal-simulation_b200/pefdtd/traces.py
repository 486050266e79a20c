"""Batched trace post-processing on the GPU: Hilbert envelope, detrend,
envelope picks and the sweep driver's per-trace analysis, float64 on the
device (csrc/pe_traces.cu through the C ABI).

The device counterparts of the reference's host helpers:
* ``envelope``    -- np.abs(scipy.signal.hilbert(x)) (sim/core/fdtd.py:976,
  sim/pipeline/sweep_runner.py:210);
* ``pick_peaks``  -- pick_peak (sim/core/fdtd.py:951-984) over many traces,
  with the same window, edge guard and parabolic refinement, detrended by
  detrend_hp (:943-948) when ``f_lo`` is given, else by the mean;
* ``analyse``     -- sweep_runner._analyse (:209-225): E1, t1, coda, tail.

Traces may differ in length (a ragged batch is packed back to back); each is
transformed over its own length, as the reference transforms each array.
Window bounds and filter coefficients are computed here on the host with the
reference's own expressions; the sample work (transforms, filters,
reductions) runs on the device. The Hilbert transform is evaluated as a
circular convolution in float64 rather than by FFT, so envelopes agree with
SciPy's to rounding (~1e-13 relative), not bit for bit.
"""
from __future__ import annotations

import numpy as np

from . import _capi


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pefdtd.traces runs on a CUDA device; the reference's host helpers "
                           "are pefdtd.wavelets.pick_peak / analyse_trace")
    return torch


def _device(torch, device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def _as_list(xs):
    if isinstance(xs, np.ndarray) and xs.ndim == 2:
        return [xs[i] for i in range(xs.shape[0])]
    try:
        import torch
        if isinstance(xs, torch.Tensor) and xs.dim() == 2:
            return list(xs.unbind(0))
    except ImportError:
        pass
    if isinstance(xs, (list, tuple)):
        return list(xs)
    return [xs]


class _Packed:
    """Traces packed back to back in one device array (f32 when every
    trace is f32, else f64) with their host offsets."""

    def __init__(self, torch, dev, xs):
        xs = _as_list(xs)
        if not xs:
            raise ValueError("no traces")
        ts = []
        for x in xs:
            if isinstance(x, torch.Tensor):
                t = x.detach().reshape(-1)
            else:
                a = np.asarray(x)
                if a.dtype != np.float32:
                    a = a.astype(np.float64)
                t = torch.from_numpy(np.ascontiguousarray(a.reshape(-1)))
            if t.numel() == 0:
                raise ValueError("empty trace")
            ts.append(t)
        f32 = all(t.dtype == torch.float32 for t in ts)
        dt = torch.float32 if f32 else torch.float64
        self.x = torch.cat([t.to(device=dev, dtype=dt) for t in ts]).contiguous()
        self.dtype = _capi.PE_F32 if f32 else _capi.PE_F64
        self.lens = np.array([t.numel() for t in ts], np.int64)
        self.off = np.zeros(len(ts) + 1, np.int64)
        np.cumsum(self.lens, out=self.off[1:])
        self.batch = len(ts)

    def split(self, y):
        yh = y.cpu().numpy()
        return [yh[self.off[i]:self.off[i + 1]] for i in range(self.batch)]


def _stream(torch, dev):
    return _capi.C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _envelope_dev(torch, dev, P, x=None, dtype=None):
    x = P.x if x is None else x
    dtype = P.dtype if dtype is None else dtype
    env = torch.empty(int(P.off[-1]), dtype=torch.float64, device=dev)
    _capi.check(_capi.lib().pe_trace_envelope(x.data_ptr(), dtype, _capi.ptr(P.off), P.batch,
                                              env.data_ptr(), _stream(torch, dev)))
    return env


def envelope(xs, device=None):
    """|hilbert(x)| of each trace (float64 numpy arrays, one per trace; a
    single array for a single 1-D input)."""
    torch = _torch()
    dev = _device(torch, device)
    single = xs.dim() == 1 if hasattr(xs, "dim") else (not isinstance(xs, (list, tuple)) and np.ndim(xs) == 1)
    with torch.cuda.device(dev):
        P = _Packed(torch, dev, xs)
        out = P.split(_envelope_dev(torch, dev, P))
    return out[0] if single else out


def _butter_hp(dt, f_lo, order=2):
    """detrend_hp's filter (sim/core/fdtd.py:943-948) and filtfilt's
    defaults: b, a normalised to a[0] = 1, lfilter_zi, padlen."""
    from scipy.signal import butter, lfilter_zi
    b, a = butter(order, f_lo / (0.5 / dt), "high")
    b, a = np.asarray(b, float), np.asarray(a, float)
    if a[0] != 1.0:
        b, a = b / a[0], a / a[0]
    n = max(len(a), len(b))
    b = np.concatenate([b, np.zeros(n - len(b))])
    a = np.concatenate([a, np.zeros(n - len(a))])
    # lfilter_zi returns a strided view: copy before handing its address on
    return b, a, np.ascontiguousarray(lfilter_zi(b, a), float), 3 * n


def detrend(xs, dt=None, f_lo=None, device=None):
    """detrend_hp(x, dt, f_lo) of each trace (Butterworth order 2 high-pass,
    filtfilt with odd padding), or x - mean(x) when f_lo is None."""
    torch = _torch()
    dev = _device(torch, device)
    with torch.cuda.device(dev):
        P = _Packed(torch, dev, xs)
        return P.split(_detrend_dev(torch, dev, P, dt, f_lo))


def _detrend_dev(torch, dev, P, dt, f_lo):
    out = torch.empty(int(P.off[-1]), dtype=torch.float64, device=dev)
    L = _capi.lib()
    if not f_lo:
        _capi.check(L.pe_trace_detrend(P.x.data_ptr(), P.dtype, _capi.ptr(P.off), P.batch, None, None, 0,
                                       None, 0, out.data_ptr(), _stream(torch, dev)))
        return out
    b, a, zi, padlen = _butter_hp(dt, f_lo)
    if int(P.lens.min()) <= padlen:
        raise ValueError(f"The length of the input vector x must be greater than padlen, which is {padlen}.")
    _capi.check(L.pe_trace_detrend(P.x.data_ptr(), P.dtype, _capi.ptr(P.off), P.batch, _capi.ptr(b),
                                   _capi.ptr(a), len(b), _capi.ptr(zi), padlen, out.data_ptr(),
                                   _stream(torch, dev)))
    return out


def pick_window(n, dt, t_end, t_lo=None, t_hi=None, edge_frac=0.04):
    """pick_peak's search window [lo, hi) (sim/core/fdtd.py:977-979)."""
    g = max(int(edge_frac * n), 4)
    lo = max(int((t_lo or 0.0) / dt), g)
    hi = min(int((t_hi or t_end) / dt), n - g)
    return lo, hi


def pick_peaks(ts, xs, t_lo=None, t_hi=None, dt=None, f_lo=None, edge_frac=0.04, device=None):
    """pick_peak(t, x, t_lo, t_hi, dt, f_lo, edge_frac) for every trace of
    ``xs``; ``ts`` is one time axis shared by all traces or one per trace.
    Returns a list of (time, envelope peak, ok)."""
    torch = _torch()
    dev = _device(torch, device)
    xl = _as_list(xs)
    tl = [np.asarray(t, float) for t in ts] if isinstance(ts, (list, tuple)) else [np.asarray(ts, float)] * len(xl)
    if len(tl) != len(xl):
        raise ValueError("one time axis per trace, or one for all")
    dts = [float(t[1] - t[0]) if dt is None else float(dt) for t in tl]
    res = [(np.nan, 0.0, False)] * len(xl)
    # one device pass per distinct time step (the filter depends on it)
    for d in sorted(set(dts)):
        idx = [i for i in range(len(xl)) if dts[i] == d]
        with torch.cuda.device(dev):
            P = _Packed(torch, dev, [xl[i] for i in idx])
            env = _envelope_dev(torch, dev, P, _detrend_dev(torch, dev, P, d, f_lo), _capi.PE_F64)
            win, keep = [], []
            for j, i in enumerate(idx):
                lo, hi = pick_window(int(P.lens[j]), d, tl[i][-1], t_lo, t_hi, edge_frac)
                if hi > lo + 2:
                    win.append((lo, hi))
                    keep.append(j)
            if not keep:
                continue
            # traces whose window is too short are settled on the host
            Q = P if len(keep) == P.batch else None
            if Q is None:
                sel = torch.cat([env[int(P.off[j]):int(P.off[j + 1])] for j in keep])
                off = np.zeros(len(keep) + 1, np.int64)
                np.cumsum(P.lens[keep], out=off[1:])
            else:
                sel, off = env, P.off
            w = np.ascontiguousarray(np.array(win, np.int64).reshape(-1))
            dv = np.full(len(keep), d)
            out = torch.empty((len(keep), 3), dtype=torch.float64, device=dev)
            _capi.check(_capi.lib().pe_trace_pick(sel.data_ptr(), _capi.ptr(off), len(keep), _capi.ptr(w),
                                                  _capi.ptr(dv), out.data_ptr(), _stream(torch, dev)))
            o = out.cpu().numpy()
        for r, j in enumerate(keep):
            res[idx[j]] = (float(o[r, 0]), float(o[r, 1]), bool(o[r, 2] != 0.0))
    return res


def analysis_windows(n, dt, path_m=0.200, c_ref=3850.0):
    """E1 window [a, b) and coda window [lo, hi) of _analyse
    (sim/pipeline/sweep_runner.py:212-218) and fs."""
    fs = 1.0 / dt
    k0 = int(path_m / c_ref * fs)
    a, b = max(k0 - int(2e-6 * fs), 0), min(k0 + int(2e-6 * fs), n)
    lo, hi = int(24e-6 * fs), min(int(36e-6 * fs), n)
    return (a, b, lo, hi), fs


def analyse(xs, dt, path_m=0.200, c_ref=3850.0, device=None):
    """(E1, t1, coda_db, tail) of every trace, as the sweep driver reports
    them; ``dt`` is one time step for all traces or one per trace."""
    torch = _torch()
    dev = _device(torch, device)
    with torch.cuda.device(dev):
        P = _Packed(torch, dev, xs)
        dts = np.broadcast_to(np.asarray(dt, float), (P.batch,))
        win = np.zeros((P.batch, 4), np.int64)
        tf = np.zeros((P.batch, 2))
        for i in range(P.batch):
            w, fs = analysis_windows(int(P.lens[i]), float(dts[i]), path_m, c_ref)
            if w[1] <= w[0]:
                raise ValueError("attempt to get argmax of an empty sequence")
            win[i], tf[i] = w, (float(dts[i]), fs)
        env = _envelope_dev(torch, dev, P)
        out = torch.empty((P.batch, 4), dtype=torch.float64, device=dev)
        _capi.check(_capi.lib().pe_trace_analyse(P.x.data_ptr(), P.dtype, env.data_ptr(), _capi.ptr(P.off),
                                                 P.batch, _capi.ptr(win), _capi.ptr(tf), out.data_ptr(),
                                                 _stream(torch, dev)))
        o = out.cpu().numpy()
    return [(float(r[0]), float(r[1]), float(r[2]), float(r[3])) for r in o]
