"""Batched solves (GPU): each solve of a mixed-size batch is bit-identical to
its own single solve and to the oracle; the autotuner leaves results
unchanged; solves the TMA kernels cannot take run in the same graph."""
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
    with pytest.raises(ValueError, match="empty"):
        batch.BatchSolver([])
    with pytest.raises(Exception, match="wavelet shorter"):
        b = batch.BatchSolver([batch.spec_from_problem(probs[0])])
        try:
            b.run(0, probs[0]["nt"] + 1)
        finally:
            b.close()


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_mixed_batch_with_unaligned_rows(dtype):
    """Solves with nx % 4 != 0 (the cp.async kernels) ride in the same graph
    as TMA-fed solves; every one stays bit-identical to the oracle."""
    from pefdtd import batch
    probs = [make_small(nt=70, shape=(16, 20, 30), n_grains=4, sponge=2, seed=3),
             make_small(nt=70, shape=(20, 28, 32), n_grains=6, sponge=3, seed=4),
             make_small(nt=70, shape=(18, 22, 27), n_grains=5, sponge=3, seed=5)]
    probs[2]["record"] = "pressure"
    b = batch.BatchSolver([batch.spec_from_problem(p) for p in probs], dtype=dtype, z_chunk=9,
                          chunk_steps=30)
    try:
        b.run(0, 70)
        got = b.traces_numpy(70)
        # 70 steps: two graph chunks and a 10-step tail; 2 + 2*2 kernels per step
        assert b.launch_count() == 70 * 6 + 3 * 3 + 3 + 1
    finally:
        b.close()
    for p, tr in zip(probs, got):
        npdt = np.dtype(dtype)
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True, dtype=npdt),
                           dtype=npdt, fma_mode=1)
        assert np.array_equal(tr, ref)


def test_batch_of_only_unaligned_rows():
    from pefdtd import batch
    probs = [make_small(nt=40, shape=(15, 19, 23), n_grains=4, sponge=2, seed=9)]
    out = batch.forward_batch(probs, autotune=False)
    ref = O.run_oracle(oracle_prob(probs[0], record=probs[0]["record"], damped_record=True), fma_mode=1)
    assert np.array_equal(out[0], ref)


def test_pair_batch_large_table_and_mixed_orders():
    """An FP32 batch whose largest table exceeds shared memory and whose
    solves mix stencil orders (the pair kernels' general instantiations)."""
    from pefdtd import batch
    from pefdtd.coeffs import optimised_coeffs
    a = dict(make_small(nt=60, shape=(14, 40, 40), n_grains=600, sponge=2, seed=21))
    b6 = dict(make_small(nt=60, shape=(16, 36, 44), n_grains=7, sponge=2, seed=22))
    b6["coeffs"] = optimised_coeffs(6)
    probs = [a, b6]
    bs = batch.BatchSolver([batch.spec_from_problem(p) for p in probs], z_chunk=5, chunk_steps=25)
    try:
        bs.run(0, 60)
        got = bs.traces_numpy(60)
    finally:
        bs.close()
    for p, tr in zip(probs, got):
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True), fma_mode=1)
        assert np.abs(ref).max() > 0
        assert np.array_equal(tr, ref)


def test_batch_mixing_solo_and_shared_solves():
    """A solve large enough to fill the GPU alone runs its own launches inside
    the batch's graph next to small solves in the shared launches; tables of
    different sizes coexist (kernel attributes are per kernel, not per solve)."""
    from pefdtd import batch
    big = make_small(nt=40, shape=(40, 256, 256), n_grains=300, sponge=4, seed=31)
    small = [make_small(nt=40, shape=(20, 28, 32), n_grains=5, sponge=3, seed=32),
             make_small(nt=40, shape=(18, 36, 40), n_grains=40, sponge=3, seed=33)]
    probs = [big] + small
    b = batch.BatchSolver([batch.spec_from_problem(p) for p in probs], chunk_steps=20)
    try:
        b.run(0, 40)
        got = b.traces_numpy(40)
    finally:
        b.close()
    for p, tr in zip(probs, got):
        ref = O.run_oracle(oracle_prob(p, record=p["record"], damped_record=True), fma_mode=1)
        assert np.abs(ref).max() > 0
        assert np.array_equal(tr, ref)


@pytest.mark.parametrize("case", ["mixed", "large_table_orders", "with_solo"])
def test_persistent_batch_equals_per_step_launches(case):
    """One cooperative launch per graph chunk (every step of the batched
    solves, grid barriers between the phases) gives the per-step launches'
    traces and final states bit for bit, on fewer launches; a partial chunk
    (not captured) too."""
    from pefdtd import batch
    from pefdtd.coeffs import optimised_coeffs
    if case == "mixed":
        probs, nt, kw = _problems(), 90, dict(z_chunk=7, chunk_steps=40)
    elif case == "large_table_orders":
        a = dict(make_small(nt=60, shape=(14, 40, 40), n_grains=600, sponge=2, seed=21))
        b6 = dict(make_small(nt=60, shape=(16, 36, 44), n_grains=7, sponge=2, seed=22))
        b6["coeffs"] = optimised_coeffs(6)
        probs, nt, kw = [a, b6], 60, dict(z_chunk=5, chunk_steps=25)
    else:
        probs = [make_small(nt=40, shape=(40, 256, 256), n_grains=300, sponge=4, seed=31),
                 make_small(nt=40, shape=(20, 28, 32), n_grains=5, sponge=3, seed=32)]
        nt, kw = 40, dict(chunk_steps=20)
    out = {}
    for persistent in (False, True):
        b = batch.BatchSolver([batch.spec_from_problem(p) for p in probs], **kw)
        try:
            assert b.set_persistent(persistent) == persistent
            b.run(0, nt - 7)
            b.run(nt - 7, nt)
            out[persistent] = (b.traces_numpy(nt), [s.cpu().numpy() for s in b.states], b.launch_count())
        finally:
            b.close()
    (t0, s0, l0), (t1, s1, l1) = out[False], out[True]
    for a, c in zip(t0, t1):
        assert np.abs(a).max() > 0
        assert np.array_equal(a, c)
    for a, c in zip(s0, s1):
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
    assert l1 < l0
