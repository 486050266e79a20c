"""Generate tests/golden/disk_prod_ref_echo.npz: the production disk's
z-velocity trace computed by the reference's own dense update kernels
(strains, stress_acc, vel_update; sim/core/fdtd.py:392-583, driven as
forward_fused drives them, :875-921), compiled for the host into oracle/_ref.

The full 160 x 256 x 256 grid (500 grains, so the dense kernels: the
reference's label path holds materials in uint8) for the first STEPS steps,
which take the trace through the transmitted burst and the disk's
bottom-face echo. On the host this is tens of minutes, too long for a test,
so the trace is kept as a fixture (7 KB) together with a digest of the inputs
it was computed from; tests/test_echo_parity_gpu.py rebuilds the inputs from
the seeded workload, checks the digest, and compares the GPU trace with it.

  python tests/golden/make_disk_prod_echo.py   (needs oracle/_ref)
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "pulse-echo-azimuthal-simulation_b200")]

STEPS = 1800
OUT = os.path.join(HERE, "disk_prod_ref_echo.npz")


def input_digest(p, prob):
    """SHA-256 over everything the trace depends on."""
    h = hashlib.sha256()
    for a in (p["mats"], np.asarray(p["Ct"], np.float32), np.asarray(p["rho_t"], np.float32),
              prob["damp"], prob["src_idx"], prob["src_w"], prob["rec_off"], prob["rec_idx"],
              prob["rec_w"], prob["wavelet"], prob["coeffs"]):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(np.float32([prob["inv_h"], prob["dt"], prob["dt_h"]]).tobytes())
    return h.hexdigest()


def main():
    from oracle import oracle as O
    from pefdtd import workloads
    p = workloads.make_problem("disk_prod", nt=STEPS, use_gpu=False)
    prob = O.problem_from_workload(p, record="vz", damped_record=True)
    t0 = time.time()
    tr = O.run_reference_dense(prob)
    el = time.time() - t0
    np.savez_compressed(OUT, trace=tr[:, 0], steps=STEPS, dt=p["dt"], digest=input_digest(p, prob),
                        seconds=el, threads=os.cpu_count())
    print(f"wrote {OUT}: {STEPS} steps in {el:.0f} s")


if __name__ == "__main__":
    main()
