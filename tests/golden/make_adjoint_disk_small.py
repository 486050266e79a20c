"""Generate tests/golden/adjoint_disk_small.npz: the reference inversion's own
gradient on the 96 x 96 x 64 copy of the gradient configuration.

The reference's only FDTD gradient is ringfwi's order-2, undamped,
cell-density adjoint (vendor/ringfwi/elastic3d.py:348-463) chained to
per-voxel c-axis angles (vendor/ringfwi/axisfield.py:123-161); it keeps the
whole velocity history in host memory. It is run here on the disk_small
specimen (64 x 96 x 96 cells at 0.2 mm, 50 Voronoi grains, the workload's
labels) in the configuration in which the two adjoints compute the same
discrete gradient: order 2 (coefficient [1.0]), no sponge, pressure record,
uniform density 917 (the couplant given the ice density, so face and cell
densities agree), explosive source. The misfit is against the traces of the
same labels with the c-axes re-drawn (the next seed). nt is reduced to 300
steps (the 1 MHz burst reaches the bottom face; ~4 GB of history) from the
workload's 2000.

Stored: the per-grain angles, the observed traces, J and the per-grain
gradients (per-voxel gradients summed over each grain), with a digest of the
labels the test rebuilds from the seeded workload.

  PE_REFERENCE_ROOT=<reference checkout> python tests/golden/make_adjoint_disk_small.py
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "adjoint_disk_small.npz")
NT = 300


def label_digest(lab):
    return hashlib.sha256(np.ascontiguousarray(lab, np.int32).tobytes()).hexdigest()


def setup(p):
    """Time step, wavelet (the reference's Hann burst) and probe of the
    matched problem for workload dict p."""
    h = p["h"]
    dt = 0.4 * h / (np.sqrt(3.0) * 4100.0)
    spec = p["spec"]
    from ringfwi import sources
    wav = sources.hann_tone_burst(NT, dt, spec["f0"], n_cycles=spec["n_cycles"])
    pts = [tuple(q) for q, _ in p["src_pts"]]
    return dt, wav, pts


def main():
    ref = os.environ.get("PE_REFERENCE_ROOT")
    if not ref or not os.path.isdir(os.path.join(ref, "vendor", "ringfwi")):
        raise SystemExit("set PE_REFERENCE_ROOT to the reference checkout (it imports vendor/ringfwi)")
    sys.path[:0] = [os.path.join(ref, "vendor"), ROOT, os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200")]
    from ringfwi import anisotropy as an
    from ringfwi import axisfield as af
    from ringfwi import elastic3d as e3
    from pefdtd import adjoint, specimen, workloads
    p = workloads.make_problem("disk_small", nt=NT, use_gpu=False)
    lab = p["lab"]
    n_g = int(lab.max()) + 1
    theta, phi = adjoint.angles_from_axes(p["axes"])
    rng = np.random.default_rng(int(p["spec"]["seed"]) + 1)
    t = np.radians(30.0)
    axes_obs = specimen.sample_watson(n_g, (np.sin(t), 0.0, np.cos(t)), 5.0, rng)
    theta_obs, phi_obs = adjoint.angles_from_axes(axes_obs)
    mask = lab >= 0
    base6 = an.ti_stiffness_6(**an.ICE_MATERIAL)
    fl = np.zeros((6, 6))
    fl[:3, :3] = 917.0 * 1500.0 ** 2
    Cbg = {k: np.full(lab.shape, fl[int(k[1]) - 1, int(k[2]) - 1]) for k in af.KEYS21}
    dt, wav, pts = setup(p)
    w = 1.0 / len(pts)
    src_pts = [[(q, w) for q in pts]]
    recs = [(pts, [w] * len(pts))]

    def maps(th, ph):
        cm = np.zeros(lab.shape)
        am = np.zeros(lab.shape)
        cm[mask] = th[lab[mask]]
        am[mask] = ph[lab[mask]]
        return cm, am

    t0 = time.time()
    co, ao = maps(theta_obs, phi_obs)
    Cobs, rho = af.build_maps(co, ao, mask, base6, Cbg, 917.0, 917.0)
    dobs, _ = e3._grad_forward(Cobs, rho, p["h"], dt, NT, None, wav, None, src_pts=src_pts[0], rec_groups=recs)
    cm, am = maps(theta, phi)
    J, g_t, g_p = af.misfit_and_gradient_axes(cm, am, mask, base6, Cbg, 917.0, 917.0, p["h"], dt, NT,
                                              src_pts, wav, recs, dobs[None])
    gt = np.array([g_t[lab == g].sum() for g in range(n_g)])
    gp = np.array([g_p[lab == g].sum() for g in range(n_g)])
    np.savez_compressed(OUT, digest=label_digest(lab), theta=theta, phi=phi, h=p["h"], dt=dt, nt=NT,
                        wavelet=wav, pts=np.array(pts), dobs=dobs, J=J, g_theta=gt, g_phi=gp,
                        seconds=time.time() - t0)
    print(f"wrote {OUT}: J {J:.6e}, |g| {np.linalg.norm(np.concatenate([gt, gp])):.3e}, "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
