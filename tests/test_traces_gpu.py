"""Device trace post-processing (pe_trace_* through the C ABI) against the
reference's host computations: scipy.signal.hilbert envelopes, detrend_hp,
pick_peak (sim/core/fdtd.py:943-984) and the sweep analysis
(sim/pipeline/sweep_runner.py:209-225), restated in pefdtd.wavelets and
pinned there. Ragged batches, f32 and f64 inputs, lengths from 1 sample.

Tolerances: the detrend filter runs the same recursion with the same
roundings as SciPy and is bit-exact; the envelope is a float64 circular
convolution instead of an FFT, so envelope values, peaks, E1 and tails agree
to 1e-11 relative, coda levels to 1e-9 dB, and pick indices and arrival
times exactly (refined times to 1e-6 of a sample)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LENS = [1, 2, 3, 8, 9, 127, 511, 512, 513, 1024, 4678, 5937, 6000]


def echo_traces(lens, dt=1e-8, seed=0, dtype=np.float64):
    """Pulse-echo-like records: a few 2 MHz tone bursts (the first near the
    2 x 100 mm round trip), a decaying coda, noise, a DC pedestal and drift."""
    rng = np.random.default_rng(seed)
    out = []
    for n in lens:
        t = np.arange(n) * dt
        x = 0.3 + 0.5 * t / max(t[-1], dt) + 0.01 * rng.standard_normal(n)
        for t0, amp in ((51.9e-6 + 0.3e-6 * rng.standard_normal(), 1.0),
                        (20e-6 * rng.random(), 0.4), (30e-6 + 10e-6 * rng.random(), 0.2)):
            tau = t - t0
            m = (tau >= 0) & (tau <= 2.5e-6)
            x[m] += amp * 0.5 * (1 - np.cos(2 * np.pi * tau[m] / 2.5e-6)) * np.sin(2 * np.pi * 2e6 * tau[m])
        x += 0.05 * np.exp(-np.maximum(t - 55e-6, 0) / 20e-6) * rng.standard_normal(n) * (t > 55e-6)
        out.append(x.astype(dtype))
    return out


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_envelope_matches_scipy_hilbert(dtype):
    from scipy.signal import hilbert
    from pefdtd import traces
    xs = echo_traces(LENS, dtype=dtype)
    env = traces.envelope(xs)
    for x, e in zip(xs, env):
        ref = np.abs(hilbert(np.asarray(x, float)))
        assert e.shape == ref.shape
        assert np.abs(e - ref).max() <= 1e-11 * max(ref.max(), 1e-300), len(x)
    one = traces.envelope(xs[-1])
    assert np.array_equal(one, env[-1])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_detrend_bit_exact_and_demean(dtype):
    from pefdtd import traces, wavelets
    xs = echo_traces([10, 11, 200, 4678, 6000], dtype=dtype)
    for dt, f_lo in ((1e-8, 0.3e6), (2e-8, 1e6)):
        got = traces.detrend(xs, dt, f_lo)
        for x, g in zip(xs, got):
            np.testing.assert_array_equal(g, wavelets.detrend_hp(np.asarray(x, float), dt, f_lo))
    got = traces.detrend(xs)
    for x, g in zip(xs, got):
        xf = np.asarray(x, float)
        assert np.abs(g - (xf - xf.mean())).max() <= 1e-14 * np.abs(xf).max()
    with pytest.raises(ValueError, match="padlen"):
        traces.detrend([np.ones(9)], 1e-8, 0.3e6)


@pytest.mark.parametrize("f_lo", [None, 0.3e6])
def test_pick_peaks_match_pick_peak(f_lo):
    from pefdtd import traces, wavelets
    dt = 1e-8
    lens = [6000, 5937, 4678, 7000, 60, 300, 6000]
    xs = echo_traces(lens, dt=dt, seed=3)
    ts = [np.arange(n) * dt for n in lens]
    for t_lo, t_hi in ((None, None), (40e-6, 60e-6), (10e-6, 45e-6), (55e-6, 55.02e-6)):
        got = traces.pick_peaks(ts, xs, t_lo=t_lo, t_hi=t_hi, f_lo=f_lo)
        for t, x, g in zip(ts, xs, got):
            ref = wavelets.pick_peak(t, x, t_lo=t_lo, t_hi=t_hi, dt=dt, f_lo=f_lo)
            assert g[2] == ref[2]
            if np.isnan(ref[0]):
                assert np.isnan(g[0]) and g[1] == ref[1] == 0.0
                continue
            assert int(round(g[0] / dt)) == int(round(ref[0] / dt))
            assert abs(g[0] - ref[0]) <= 1e-6 * dt
            assert abs(g[1] - ref[1]) <= 1e-11 * ref[1]
    # one time axis shared by every trace (same length)
    xs2 = echo_traces([6000] * 4, dt=dt, seed=9)
    t = np.arange(6000) * dt
    got = traces.pick_peaks(t, xs2, t_lo=30e-6, f_lo=f_lo)
    for x, g in zip(xs2, got):
        ref = wavelets.pick_peak(t, x, t_lo=30e-6, dt=dt, f_lo=f_lo)
        assert abs(g[0] - ref[0]) <= 1e-6 * dt and g[2] == ref[2]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_analyse_matches_sweep_analysis(dtype):
    from pefdtd import traces, wavelets
    dt = 1e-8
    lens = [6000, 5937, 7000, 5500, 5300, 9895]     # 5500, 5300: record ends before the tail window
    xs = echo_traces(lens, dt=dt, seed=5, dtype=dtype)
    got = traces.analyse(xs, dt)
    for x, g in zip(xs, got):
        ref = wavelets.analyse_trace(np.asarray(x, float), dt, path_m=0.200, c_ref=3850.0)
        assert abs(g[0] - ref[0]) <= 1e-11 * ref[0]
        assert g[1] == ref[1]
        assert abs(g[2] - ref[2]) <= 1e-9
        if np.isnan(ref[3]):
            assert np.isnan(g[3])
        else:
            assert abs(g[3] - ref[3]) <= 1e-11 * ref[3]
    assert np.isnan(got[3][3]) and np.isnan(got[4][3])
    # per-trace time steps
    dts = [1e-8, 1.2e-8, 0.9e-8]
    xs3 = [echo_traces([n], dt=d, seed=k)[0] for k, (n, d) in enumerate(zip((6000, 5000, 7000), dts))]
    got = traces.analyse(xs3, dts)
    for x, d, g in zip(xs3, dts, got):
        ref = wavelets.analyse_trace(x, d, path_m=0.200, c_ref=3850.0)
        assert g[1] == ref[1] and abs(g[0] - ref[0]) <= 1e-11 * ref[0]
