"""CPU checks of the algorithms the device trace kernels evaluate
(csrc/pe_traces.cu): the closed-form discrete Hilbert kernel and the
filtfilt recursion, each restated here in NumPy / plain Python and held
against SciPy, which the reference calls (sim/core/fdtd.py:943-984,
sim/pipeline/sweep_runner.py:209-225)."""
import numpy as np
import pytest

scipy_signal = pytest.importorskip("scipy.signal")


def hilbert_kernel(N):
    m = np.arange(N)
    g = np.zeros(N)
    nz = m > 0
    s, c = np.sin(np.pi * m[nz] / N), np.cos(np.pi * m[nz] / N)
    if N % 2 == 0:
        g[nz] = np.where(m[nz] % 2 == 1, (2.0 / N) * (c / s), 0.0)
    else:
        g[nz] = ((c - np.where(m[nz] % 2 == 1, -1.0, 1.0)) / s) / N
    return g


@pytest.mark.parametrize("N", [1, 2, 3, 4, 7, 8, 33, 64, 257, 1000, 1001])
def test_circular_hilbert_kernel_matches_scipy_hilbert(N):
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N)
    g = hilbert_kernel(N)
    n = np.arange(N)
    y = np.array([np.dot(x, g[(k - n) % N]) for k in range(N)])
    ref = scipy_signal.hilbert(x)
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(y - ref.imag).max() <= 1e-12 * scale
    assert np.abs(np.hypot(x, y) - np.abs(ref)).max() <= 1e-12 * scale


def _df2t(b, a, z, xs):
    """lfilter's transposed direct form II, one product per rounding."""
    out = []
    n = len(b)
    for xv in xs:
        y = z[0] + b[0] * xv
        for k in range(n - 2):
            z[k] = (z[k + 1] + xv * b[k + 1]) - y * a[k + 1]
        z[n - 2] = xv * b[n - 1] - y * a[n - 1]
        out.append(y)
    return out


def _filtfilt_restated(b, a, zi, p, x):
    N = len(x)
    ext = ([2.0 * x[0] - x[p - e] for e in range(p)] + list(x)
           + [2.0 * x[N - 1] - x[N - 2 - j] for j in range(p)])
    y = _df2t(b, a, [v * ext[0] for v in zi], ext)
    y = _df2t(b, a, [v * y[-1] for v in zi], y[::-1])[::-1]
    return np.array(y[p:p + N])


@pytest.mark.parametrize("n,dt,f_lo", [(10, 2e-8, 0.3e6), (200, 2e-8, 0.3e6), (1500, 1e-8, 0.5e6),
                                       (777, 3e-8, 1e6)])
def test_filtfilt_recursion_matches_scipy_detrend(n, dt, f_lo):
    from pefdtd import traces, wavelets
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 3.0 + np.linspace(0, 2, n)
    b, a, zi, padlen = traces._butter_hp(dt, f_lo)
    assert padlen == 9 and len(b) == len(a) == 3
    got = _filtfilt_restated(list(b), list(a), list(zi), padlen, x)
    ref = wavelets.detrend_hp(x, dt, f_lo)
    np.testing.assert_array_equal(got, ref)   # same recursion, same roundings


def test_windows_follow_the_reference_expressions():
    from pefdtd import traces
    n, dt = 6000, 1e-8
    assert traces.pick_window(n, dt, (n - 1) * dt, 10e-6, 40e-6) == (1000, 4000)
    assert traces.pick_window(n, dt, (n - 1) * dt) == (240, 5760)
    assert traces.pick_window(50, dt, 49 * dt) == (4, 46)
    (a, b, lo, hi), fs = traces.analysis_windows(n, dt)
    k0 = int(0.200 / 3850.0 * (1.0 / dt))
    assert (a, b) == (k0 - 200, k0 + 200) and (lo, hi) == (2400, 3600) and fs == 1.0 / dt
    (a, b, lo, hi), _ = traces.analysis_windows(3000, dt)
    assert b == 3000 and hi == 3000
