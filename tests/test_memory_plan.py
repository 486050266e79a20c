"""The gradient memory plan (pefdtd.adjoint: adjoint_bytes, plan_memory,
plan_waves) on the CPU: byte counts of one-level, two-level and offloaded
checkpointing, the choice for a budget, and waves that fit it."""
import numpy as np
import pytest

from helpers import make_small

DISK_PROD = (160, 256, 256)


def test_adjoint_bytes_for_the_gradient_configuration():
    from pefdtd import adjoint
    field = 4 * int(np.prod(DISK_PROD))
    one = adjoint.adjoint_bytes(DISK_PROD, 6000, 200)
    # 30 outer checkpoints of 9 fields, 200 steps of 3-field history, the
    # solver's 9 fields + labels, the adjoint state and its 33-field scratch
    assert one == 9 * field + 2 * field // 4 + 30 * 9 * field + 200 * 3 * field + 42 * field
    two = adjoint.adjoint_bytes(DISK_PROD, 6000, 200, inner_every=24)
    off = adjoint.adjoint_bytes(DISK_PROD, 6000, 200, inner_every=24, offload=True)
    assert off < two < one
    assert two == one - 200 * 3 * field + 24 * 3 * field + 9 * 9 * field   # 9 inner checkpoints
    assert off == two - 30 * 9 * field
    assert one > 35e9 and off < 10e9


def test_plan_memory_prefers_no_recomputation_then_two_levels_then_offload():
    from pefdtd import adjoint
    one = adjoint.adjoint_bytes(DISK_PROD, 6000, 200)
    assert adjoint.plan_memory(DISK_PROD, 6000, one) == (None, False)
    inner, off = adjoint.plan_memory(DISK_PROD, 6000, one - 1)
    assert inner == int(round(np.sqrt(3 * 200))) and off is False
    two = adjoint.adjoint_bytes(DISK_PROD, 6000, 200, inner_every=inner)
    got = adjoint.plan_memory(DISK_PROD, 6000, two - 1)
    assert got[1] is True
    assert adjoint.plan_memory(DISK_PROD, 6000, 1 << 20) is None


def _problems(n):
    from pefdtd.adjoint import Problem
    out = []
    for k in range(n):
        p = make_small(nt=60, shape=(16, 20, 24), n_grains=4, sponge=3, seed=50 + k)
        out.append(Problem(p["mats"], p["rho_t"], p["h"], p["dt"], p["coeffs"], p["src_pts"], p["rec_groups"],
                           p["wavelet"], record="vz", sponge_width=p["sponge"], dtype="float32",
                           checkpoint_every=20))
    return out


def test_plan_waves_fit_the_budget_and_replan_large_solves():
    from pefdtd import adjoint
    probs = _problems(5)
    each = adjoint.adjoint_bytes((16, 20, 24), 60, 20)
    assert [len(w) for w in adjoint.plan_waves(probs, 10 * each)] == [5]
    waves = adjoint.plan_waves(probs, int(2.5 * each))
    assert [len(w) for w in waves] == [2, 2, 1]
    assert [i for w in waves for i, _ in w] == list(range(5))
    assert all(opt == (None, False) for w in waves for _, opt in w)
    # below one plain solve: every solve re-planned, one per wave
    small = adjoint.plan_waves(probs, each - 1)
    assert [len(w) for w in small] == [1] * 5
    assert all(opt[0] is not None and opt[0] < 20 for w in small for _, opt in w)
    with pytest.raises(MemoryError):
        adjoint.plan_waves(probs, 1 << 10)
    # without planning an oversized solve still gets its own wave
    assert [len(w) for w in adjoint.plan_waves(probs, each - 1, plan=False)] == [1] * 5
