"""Gradients at scale and the fabric inversion (GPU).

* Two-level checkpointing (inner_every) and host-offloaded checkpoints give
  the one-level gradient (to the rounding of the f64 atomic gradient sums).
* misfit_gradients in several memory waves gives the one-wave results.
* The batched fabric inversion (pefdtd.inversion) evaluates the same misfit
  and angle gradient as the plain one-solve-at-a-time loop, the angle
  gradient matches central differences of the misfit, and L-BFGS lowers the
  misfit.
"""
import numpy as np
import pytest

from helpers import make_small, small_spec

pytestmark = pytest.mark.gpu


def _problem(p, K, dtype="float64", **kw):
    from pefdtd.adjoint import Problem
    return Problem(p["mats"], p["rho_t"], p["h"], p["dt"], p["coeffs"], p["src_pts"], p["rec_groups"],
                   p["wavelet"], record="vz", sponge_width=p["sponge"], damped_record=True, dtype=dtype,
                   checkpoint_every=K, **kw)


def _c21(p):
    from pefdtd.fdtd import _material_tables64
    from pefdtd.materials import c36_to_c21
    return c36_to_c21(_material_tables64(p["axes"], 1500.0, 300.0)[0])


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_two_level_and_offloaded_checkpoints_equal_one_level(dtype):
    from pefdtd.adjoint import misfit_gradients
    p = make_small(nt=90, shape=(18, 22, 24), n_grains=5, sponge=3, seed=41)
    c = _c21(p)
    d = _problem(p, 30, dtype).traces_numpy(c * 1.01)
    ref = misfit_gradients([_problem(p, 30, dtype)], [c], [d], plan=False)[0]
    for kw in (dict(inner_every=7), dict(offload=True), dict(inner_every=4, offload=True)):
        J, g = misfit_gradients([_problem(p, 30, dtype, **kw)], [c], [d], plan=False)[0]
        assert abs(J - ref[0]) <= 1e-13 * abs(ref[0])
        assert np.abs(g - ref[1]).max() <= 1e-10 * np.abs(ref[1]).max(), kw


def test_memory_waves_and_plan():
    from pefdtd import adjoint
    probs, c21s, dobs = [], [], []
    for k in range(5):
        p = make_small(nt=60, shape=(16, 20, 24), n_grains=4, sponge=3, seed=50 + k)
        pr = _problem(p, 20, "float32")
        probs.append(pr)
        c21s.append(_c21(p))
        dobs.append(pr.traces_numpy(c21s[-1] * 0.99))
    one = adjoint.misfit_gradients(probs, c21s, dobs, memory_budget=1 << 40)
    each = adjoint.adjoint_bytes((16, 20, 24), 60, 20)
    waves = adjoint.plan_waves(probs, int(2.5 * each))
    assert [len(w) for w in waves] == [2, 2, 1]
    got = adjoint.misfit_gradients(probs, c21s, dobs, memory_budget=int(2.5 * each))
    for (J, g), (Jr, gr) in zip(got, one):
        assert abs(J - Jr) <= 1e-13 * abs(Jr)
        assert np.abs(g - gr).max() <= 1e-10 * np.abs(gr).max()
    # a budget below one plain solve: two-level checkpoints, then host offload
    inner, off = adjoint.plan_memory((16, 20, 24), 60, each - 1, 20)
    assert inner is not None and inner < 20
    small = adjoint.misfit_gradients(probs[:1], c21s[:1], dobs[:1], memory_budget=each - 1)[0]
    assert np.abs(small[1] - one[0][1]).max() <= 1e-10 * np.abs(one[0][1]).max()


def _inversion(batched):
    from pefdtd import inversion
    specs = [small_spec(shape=(18, 22, 24), n_grains=5, seed=61, nt=120, sponge=3),
             small_spec(shape=(16, 24, 24), n_grains=4, seed=62, nt=120, sponge=3)]
    disks = [inversion.Disk(s, [0.0, 40.0, 130.0], nt=120, dtype="float64", checkpoint_every=40)
             for s in specs]
    d_obs = inversion.observe(disks)
    rng = np.random.default_rng(5)
    x0 = np.concatenate([a for d in disks for a in inversion.isotropic_angles(d.n_grains, rng)])
    return inversion.FabricInversion(disks, d_obs, batched=batched), x0, disks


def test_batched_inversion_equals_plain_and_descends():
    inv_b, x0, disks = _inversion(True)
    inv_p, _, _ = _inversion(False)
    Jb, gb = inv_b.objective(x0)
    Jp, gp = inv_p.objective(x0)
    assert Jb > 0 and abs(Jb - Jp) <= 1e-12 * Jp
    assert np.abs(gb - gp).max() <= 1e-9 * np.abs(gp).max()
    # the angle gradient against central differences of the misfit
    rng = np.random.default_rng(9)
    for i in rng.choice(len(x0), size=3, replace=False):
        h = 1e-4
        xp, xm = x0.copy(), x0.copy()
        xp[i] += h
        xm[i] -= h
        fd = (inv_b.objective(xp)[0] - inv_b.objective(xm)[0]) / (2 * h)
        assert abs(fd - gb[i]) <= 1e-4 * np.abs(gb).max(), (i, fd, gb[i])
    res = inv_b.run(x0, iterations=3)
    assert res["iterations"] >= 1 and res["J"] < res["J0"]
