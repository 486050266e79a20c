"""Solves dealt to ranks (pefdtd.shard) and the sharded sweep, as two gloo
ranks on the CPU. The solver is a stand-in (the GPU solve is covered by the
GPU tests); what is checked is who solves what and that every rank ends with
every trace, in input order."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np

from helpers import synthetic_echo  # noqa: F401  (puts the package on sys.path)
from pefdtd import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assign_is_a_balanced_partition():
    rng = np.random.default_rng(3)
    costs = rng.uniform(1, 10, size=37)
    for world in (1, 2, 3, 8):
        shares = shard.assign(costs, world)
        assert sorted(i for s in shares for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert shares == shard.assign(costs, world)   # every rank computes the same shares
    # uneven grids: the two heaviest solves land on different ranks (loads 7 and 6)
    assert shard.assign([5, 1, 1, 1, 4, 1], 2) == [[0, 2, 5], [1, 3, 4]]


def _worker(rank, world, port, out_dir, mode):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        if mode == "traces":
            items = list(range(11))
            costs = [1 + (i % 4) for i in items]
            solved = []

            def solver(xs):
                solved.extend(xs)
                return [np.full(3, 1.5 * x) for x in xs]
            out = shard.run_sharded(items, solver, costs=costs)
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"solved": solved, "out": [list(map(float, t)) for t in out]}, f)
        else:
            from pefdtd import sweep
            from test_sweep import CFG
            if rank == 0:
                sweep.create("shard", out_dir, **CFG)
            dist.barrier()
            cfg = sweep.load("shard", out_dir)

            def solver(setups, progress):
                progress(1.0)
                return [synthetic_echo(s["nt"], s["dt"], s["f0"]).astype(float) for s in setups]
            if rank == 1:
                # start late: a rank that read the pending azimuths on its
                # own after rank 0 had written its share would shard a
                # shorter list, and azimuths would go unsolved
                import time
                time.sleep(3.0)
            res = sweep.run(cfg, labeller="exact", batch=2, log=lambda *a: None, solver=solver,
                            prefetch=False, rank=rank, world=world)
            dist.barrier()
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"result": res}, f)
    finally:
        dist.destroy_process_group()


def _spawn(tmp_path, mode, world=2):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), mode)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return [json.load(open(os.path.join(tmp_path, f"r{r}.json"))) for r in range(world)]


def test_run_sharded_gloo_two_ranks(tmp_path):
    res = _spawn(tmp_path, "traces")
    items = list(range(11))
    shares = shard.assign([1 + (i % 4) for i in items], 2)
    for r in range(2):
        assert res[r]["solved"] == shares[r]          # each rank solved its share only
        assert res[r]["out"] == [[1.5 * i] * 3 for i in items]   # and holds every trace


def test_sharded_sweep_gloo_two_ranks(tmp_path):
    """Two ranks split the pending azimuths of one sweep, rank 1 starting
    late; together they write every az file once, and the sweep is complete
    for both."""
    from pefdtd import sweep
    res = _spawn(tmp_path, "sweep")
    assert [r["result"] for r in res] == ["complete", "complete"]
    cfg = sweep.load("shard", str(tmp_path))
    assert sweep.done_azimuths(cfg, str(tmp_path)) == sorted(sweep.azimuths(cfg))
    assert sweep.pending(cfg, str(tmp_path)) == []
