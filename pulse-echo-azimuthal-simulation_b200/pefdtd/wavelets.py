"""Source wavelets and echo picking.

ricker: sim/core/fdtd.py:925-940 (t0 = 1.2 / f0).
hann_tone_burst: vendor/ringfwi/sources.py:45-60.
detrend_hp / pick_peak: sim/core/fdtd.py:943-984 — the Hilbert-envelope pick
that defines "identical echo arrival picks".
analyse_trace: sim/pipeline/sweep_runner.py:209-225 (E1, arrival, coda, tail).
"""
from __future__ import annotations

import numpy as np


def ricker(f0, dt, nt, t0=None):
    t0 = t0 if t0 is not None else 1.2 / f0
    t = np.arange(nt) * dt - t0
    a = (np.pi * f0 * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def hann_tone_burst(nt, dt, f0, n_cycles=1, t0=None):
    if t0 is None:
        t0 = 0.0
    t = np.arange(nt) * dt
    dur = n_cycles / f0
    w = np.zeros(nt)
    m = (t >= t0) & (t <= t0 + dur)
    tau = t[m] - t0
    w[m] = 0.5 * (1.0 - np.cos(2.0 * np.pi * tau / dur)) * np.sin(2.0 * np.pi * f0 * tau)
    return w


def detrend_hp(x, dt, f_lo, order=2):
    from scipy.signal import butter, filtfilt
    b, a = butter(order, f_lo / (0.5 / dt), "high")
    return filtfilt(b, a, np.asarray(x, float))


def pick_peak(t, x, t_lo=None, t_hi=None, dt=None, f_lo=None, edge_frac=0.04):
    """Envelope peak in [t_lo, t_hi] with edge guards and parabolic refinement.

    Returns (time, envelope peak, ok) where ok is False when the maximum sits
    on a window edge."""
    from scipy.signal import hilbert
    x = np.asarray(x, float)
    n = len(x)
    if dt is None:
        dt = float(t[1] - t[0])
    x = detrend_hp(x, dt, f_lo) if f_lo else x - x.mean()
    e = np.abs(hilbert(x))
    g = max(int(edge_frac * n), 4)
    lo = max(int((t_lo or 0.0) / dt), g)
    hi = min(int((t_hi or t[-1]) / dt), n - g)
    if hi <= lo + 2:
        return np.nan, 0.0, False
    k = int(np.argmax(e[lo:hi]))
    ok = 0 < k < (hi - lo - 1)
    kk = lo + k
    if 0 < kk < n - 1:
        y0, y1, y2 = e[kk - 1], e[kk], e[kk + 1]
        d = y0 - 2 * y1 + y2
        kk = kk + (0.5 * (y0 - y2) / d if abs(d) > 1e-30 else 0.0)
    return kk * dt, float(e[lo:hi].max()), ok


def analyse_trace(tr, dt, path_m=0.200, c_ref=3850.0):
    """(E1, t1, coda_db, tail) as the sweep driver reports them."""
    from scipy.signal import hilbert
    tr = np.asarray(tr, float)
    e = np.abs(hilbert(tr))
    fs = 1.0 / dt
    k0 = int(path_m / c_ref * fs)
    a, b = max(k0 - int(2e-6 * fs), 0), min(k0 + int(2e-6 * fs), len(e))
    k = a + int(np.argmax(e[a:b]))
    E1, t1 = float(e[k]), k * dt
    lo, hi = int(24e-6 * fs), min(int(36e-6 * fs), len(e))
    coda = 20 * np.log10(np.sqrt((e[lo:hi] ** 2).mean()) / E1 + 1e-30)
    k_tail = int((t1 + 3e-6) * fs)
    tail = (float(np.abs(tr[k_tail:]).max() / max(E1, 1e-30))
            if k_tail < len(tr) - 8 else float("nan"))
    return E1, t1, float(coda), tail
