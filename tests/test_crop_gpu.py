"""The causal crop on the GPU: a monostatic rim probe's trace up to t_keep is
unchanged to within -70 dB (the reference's acceptance,
sim/fw_checks/fw_crop_validate.py) when every cell beyond the causal radius
is cut away, at a fraction of the cost."""
import numpy as np
import pytest

from helpers import synthetic_echo  # noqa: F401

pytestmark = pytest.mark.gpu


def test_causal_crop_trace_within_minus_70_db():
    from scipy.signal import hilbert
    from pefdtd import crop, damping, fdtd, sweep, workloads
    spec = dict(shape=(40, 120, 200), h=0.1e-3, diameter=11e-3, height=3e-3, n_grains=14,
                fabric=("watson", 30.0, 5.0), f0=2e6, n_cycles=3, nt=700, sponge=6, aperture=2e-3, seed=4)
    p = workloads.make_problem(spec, use_gpu=False)
    lab, h, dt = p["lab"], p["h"], p["dt"]
    nd = int(round(spec["diameter"] / h))
    # rim probe on the +x side: the reference's monostatic geometry
    nz, ny, nx = lab.shape
    cz, cy, cx = nz // 2, ny // 2, nx // 2
    ks = [k for k in range(nd // 2 - 1, 0, -1) if lab[cz, cy, cx + k] >= 0]
    ixp = cx + ks[0] - 1
    er = 8
    pts = [(cz + a, cy + b, ixp) for a in range(-er, er + 1) for b in range(-er, er + 1)
           if a * a + b * b <= er * er and 0 <= cz + a < nz and lab[cz + a, cy + b, ixp] >= 0]
    w = 1.0 / len(pts)
    dm = damping.fluid_damp_mask(lab, 0.02)
    nt = 700
    wav = np.asarray(p["wavelet"][:nt])
    t_keep = nt * dt
    full = fdtd.forward_fused_labels(lab, p["axes"], h, dt, nt, [(q, w) for q in pts], wav,
                                     [(pts, np.full(len(pts), w))], coeffs=p["coeffs"],
                                     sponge_width=6, damp_mask=dm).ravel().astype(float)
    c = crop.causal_crop(lab, pts, h, dt, t_keep, damp_mask=dm)
    assert c["lab"].size < 0.75 * lab.size
    cut = fdtd.forward_fused_labels(c["lab"], p["axes"], h, dt, c["nt"], [(q, w) for q in c["pts"]], wav,
                                    [(c["pts"], np.full(len(c["pts"]), w))], coeffs=p["coeffs"],
                                    sponge_width=6, damp_mask=c["damp_mask"]).ravel().astype(float)
    n = min(len(full), len(cut))
    env_d = np.abs(hilbert(cut[:n] - full[:n]))
    env_f = np.abs(hilbert(full[:n]))
    assert 20 * np.log10(env_d.max() / env_f.max() + 1e-30) <= -70.0
