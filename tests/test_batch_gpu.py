"""Batched solves (GPU): each solve of a mixed-size batch is bit-identical to
its own single solve and to the oracle; the autotuner leaves results
unchanged; the batch refuses what it cannot run."""
import numpy as np
import pytest

from helpers import make_small, oracle_prob
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _problems():
    shapes = [(20, 28, 32), (26, 40, 48), (17, 33, 36), (22, 24, 64)]
    out = []
    for i, s in enumerate(shapes):
        p = make_small(nt=90, shape=s, n_grains=6 + 3 * i, sponge=3, seed=11 + i)
        if i == 2:
            p["record"] = "pressure"
        out.append(p)
    return out


def test_batch_matches_oracle_and_single_solves():
    from pefdtd import batch, fdtd
    probs = _problems()
    specs = [batch.spec_from_problem(p) for p in probs]
    b = batch.BatchSolver(specs, z_chunk=7, chunk_steps=40)
    try:
        b.run(0, 90)
        got = b.traces_numpy(90)
        assert b.launch_count() > 0
    finally:
        b.close()
    for p, tr in zip(probs, got):
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True), fma_mode=1)
        assert np.array_equal(tr, ref)
        single = fdtd.forward_fused_labels(p["lab"], p["axes"], p["h"], p["dt"], p["nt"], p["src_pts"],
                                           p["wavelet"], p["rec_groups"], coeffs=p["coeffs"],
                                           sponge_width=p["sponge"], record=p["record"],
                                           damped_record=True)
        assert np.array_equal(tr, single)


def test_autotune_then_run_is_unchanged(tmp_path, monkeypatch):
    monkeypatch.setenv("PEFDTD_CACHE", str(tmp_path))
    from pefdtd import autotune, batch
    probs = _problems()[:2]
    specs = [batch.spec_from_problem(p) for p in probs]
    b = batch.BatchSolver(specs)
    try:
        res = autotune.tune_batch(b)
        assert res["z_chunk"] in autotune.Z_CANDIDATES
        b.run(0, 90)
        got = b.traces_numpy(90)
        again = autotune.tune_batch(b)          # served from the cache
        assert again["z_chunk"] == res["z_chunk"]
    finally:
        b.close()
    for p, tr in zip(probs, got):
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True), fma_mode=1)
        assert np.array_equal(tr, ref)


def test_forward_batch_convenience_and_refusals():
    from pefdtd import batch
    probs = _problems()[:3]
    out = batch.forward_batch(probs, autotune=False)
    for p, tr in zip(probs, out):
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True), fma_mode=1)
        assert np.array_equal(tr, ref)
    bad = make_small(nt=20, shape=(16, 20, 30), n_grains=4, sponge=2)   # nx % 4 != 0
    with pytest.raises(Exception, match="multiple of 4"):
        batch.BatchSolver([batch.spec_from_problem(bad)])
