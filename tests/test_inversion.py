"""The fabric inversion's host logic (pefdtd.inversion) on the CPU: label
rotation, the chain from per-solve table gradients to per-grain angles
(central differences), and the same L-BFGS steps with the solves dealt over
two gloo ranks as in one process. The solver is a stand-in with a table-space
misfit (the GPU solve and its adjoint are covered by the GPU tests)."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np

from helpers import small_spec  # noqa: F401  (puts the package on sys.path)

AZ = [0.0, 90.0, 200.0]


def _disks():
    from pefdtd import inversion
    specs = [small_spec(shape=(16, 20, 24), n_grains=5, seed=3, nt=20),
             small_spec(shape=(14, 22, 22), n_grains=4, seed=8, nt=20)]
    return [inversion.Disk(s, AZ, nt=20, use_gpu=False) for s in specs]


def _stand_in(disks):
    """misfit_fn with J = 0.5 ||(c21 - T) / 1e9||^2 per solve, T the table of
    the true axes at that azimuth."""
    import torch
    from pefdtd import adjoint, inversion
    target = {}
    for d in disks:
        th, ph = adjoint.angles_from_axes(d.true_axes)
        for az, p in zip(d.azimuths, d.problems):
            target[id(p)] = inversion.tables21(torch.as_tensor(th), torch.as_tensor(ph), az).numpy()

    def fn(problems, c21s, dobs):
        out = []
        for p, c in zip(problems, c21s):
            r = (np.asarray(c) - target[id(p)]) / 1e9
            out.append((0.5 * float((r * r).sum()), r / 1e9))
        return out
    return fn


def _x0(disks):
    from pefdtd import inversion
    rng = np.random.default_rng(4)
    parts = []
    for d in disks:
        th, ph = inversion.isotropic_angles(d.n_grains, rng)
        parts += [th, ph]
    return np.concatenate(parts)


def test_rotate_labels_quarter_turns_are_exact():
    from pefdtd import inversion
    rng = np.random.default_rng(1)
    lab = rng.integers(-1, 9, size=(3, 6, 6)).astype(np.int32)
    assert np.array_equal(inversion.rotate_labels(lab, 0.0), lab)
    r90 = inversion.rotate_labels(lab, 90.0)
    # sampling rotated by +90 deg about the centre: out[y, x] = lab[x, -y] (centred indices)
    assert np.array_equal(r90, np.rot90(lab, k=1, axes=(1, 2)))
    assert np.array_equal(inversion.rotate_labels(r90, 270.0), lab)


def test_objective_gradient_matches_central_differences():
    from pefdtd import inversion
    disks = _disks()
    inv = inversion.FabricInversion(disks, [[None] * len(AZ)] * len(disks), misfit_fn=_stand_in(disks))
    x = _x0(disks)
    J, g = inv.objective(x)
    assert J > 0 and g.shape == x.shape
    rng = np.random.default_rng(2)
    for i in rng.choice(len(x), size=6, replace=False):
        h = 1e-6
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (inv.objective(xp)[0] - inv.objective(xm)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from pefdtd import inversion
        disks = _disks()
        solved = []
        fn = _stand_in(disks)

        def counting(problems, c21s, dobs):
            solved.extend(id(p) for p in problems)
            return fn(problems, c21s, dobs)
        inv = inversion.FabricInversion(disks, [[None] * len(AZ)] * len(disks), misfit_fn=counting)
        J0, g0 = inv.objective(_x0(disks))
        n0 = len(solved)
        res = inv.run(_x0(disks), iterations=3)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"J0": J0, "g0": g0.tolist(), "x": res["x"].tolist(), "J": res["J"],
                       "mine": [list(m) for m in inv.mine], "n0": n0}, f)
    finally:
        dist.destroy_process_group()


def test_sharded_inversion_gloo_two_ranks_takes_the_same_steps(tmp_path):
    from pefdtd import inversion
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [json.load(open(os.path.join(tmp_path, f"r{r}.json"))) for r in range(2)]
    # the six solves split between the ranks, none twice
    jobs = sorted(tuple(m) for r in res for m in r["mine"])
    assert jobs == [(k, a) for k in range(2) for a in range(len(AZ))]
    assert all(r["n0"] > 0 for r in res)
    # one process, all solves
    disks = _disks()
    inv = inversion.FabricInversion(disks, [[None] * len(AZ)] * len(disks), misfit_fn=_stand_in(disks))
    J0, g0 = inv.objective(_x0(disks))
    one = inv.run(_x0(disks), iterations=3)
    for r in res:
        assert abs(r["J0"] - J0) <= 1e-12 * J0
        assert np.allclose(r["g0"], g0, rtol=1e-10, atol=1e-12 * np.abs(g0).max())
        assert np.allclose(r["x"], one["x"], rtol=1e-8, atol=1e-10)
    assert res[0]["x"] == res[1]["x"]            # both ranks took identical steps
    assert one["J"] < 0.75 * J0                  # and the misfit went down
