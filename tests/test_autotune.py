"""The batch schedule autotuner's choices (pefdtd.autotune) on the CPU, with
a stand-in batch and a synthetic cost per step in place of the device
timing: the cheapest z-chunk, graph length and launch mode are chosen and
applied, candidates the batch cannot use are skipped, the batch is left
reset, and results are cached per device and batch signature."""
import types

import numpy as np
import pytest

import helpers  # noqa: F401  (puts the package on sys.path)


class FakeBatch:
    def __init__(self, shapes, nt, persistent_ok=True):
        self.shapes = shapes
        self.nt = nt
        self.npdt = np.float32
        self.device = 0
        self.torch = types.SimpleNamespace(cuda=types.SimpleNamespace(get_device_name=lambda d: "FAKE B200"))
        self.z, self.c, self.persistent = None, None, False
        self.persistent_ok = persistent_ok
        self.log = []

    def schedule(self, z, c):
        self.z, self.c = z, c
        self.log.append(("schedule", z, c))

    def set_persistent(self, on):
        if on and not self.persistent_ok:
            return False
        self.persistent = bool(on)
        self.log.append(("persistent", self.persistent))
        return True

    def reset(self):
        self.log.append(("reset",))


def cost(batch, steps):
    """ms per step: best at z = 40 and graphs of 200 steps; persistent 10 % faster."""
    c = 1.0 + 0.01 * abs(batch.z - 40) + (0.0 if batch.c in (1, None) else 0.002 * abs(batch.c - 200) / 100)
    return c * (0.9 if batch.persistent else 1.0)


@pytest.fixture
def tuner(monkeypatch, tmp_path):
    from pefdtd import autotune
    monkeypatch.setenv("PEFDTD_CACHE", str(tmp_path))
    calls = []

    def fake_time(batch, steps, warmup=2):
        calls.append((batch.z, batch.c, batch.persistent, steps))
        return cost(batch, steps)
    monkeypatch.setattr(autotune, "time_steps", fake_time)
    return autotune, calls


def test_chooses_and_applies_the_cheapest_schedule(tuner):
    autotune, calls = tuner
    b = FakeBatch([(160, 256, 256), (64, 96, 96)], nt=[600, 600])
    res = autotune.tune_batch(b)
    assert (res["z_chunk"], res["chunk_steps"], res["persistent"]) == (40, 200, True)
    assert (b.z, b.c, b.persistent) == (40, 200, True)           # applied to the batch
    assert set(res["ms_per_step_by_z"]) == set(autotune.Z_CANDIDATES)   # 160 planes: every z fits
    assert set(res["ms_per_step_by_chunk"]) == set(autotune.CHUNK_CANDIDATES)   # 600 steps: every length fits
    n_trials = len(res["ms_per_step_by_z"]) + len(res["ms_per_step_by_chunk"]) + 1
    assert b.log.count(("reset",)) == n_trials                    # every timed trial is undone


def test_skips_what_the_batch_cannot_use(tuner):
    autotune, calls = tuner
    b = FakeBatch([(48, 64, 64)], nt=[150], persistent_ok=False)
    res = autotune.tune_batch(b)
    assert set(res["ms_per_step_by_z"]) == {z for z in autotune.Z_CANDIDATES if z <= 48} | {autotune.Z_CANDIDATES[0]}
    assert set(res["ms_per_step_by_chunk"]) == {c for c in autotune.CHUNK_CANDIDATES if c + 2 <= 150}
    assert res["persistent"] is False and res["ms_per_step_by_mode"] == {} and not b.persistent


def test_results_are_cached_per_device_and_signature(tuner):
    autotune, calls = tuner
    b = FakeBatch([(160, 256, 256)], nt=[600])
    first = autotune.tune_batch(b)
    n = len(calls)
    b2 = FakeBatch([(160, 256, 256)], nt=[600])
    again = autotune.tune_batch(b2)
    assert len(calls) == n                                        # served from the cache
    assert (b2.z, b2.c, b2.persistent) == (first["z_chunk"], first["chunk_steps"], first["persistent"])
    assert again["z_chunk"] == first["z_chunk"]
    other = FakeBatch([(160, 256, 256), (160, 256, 256)], nt=[600, 600])
    autotune.tune_batch(other)
    assert len(calls) > n                                         # another signature is tuned
    # an entry cached before the launch mode was a choice is tuned again
    db = autotune._load()
    key = autotune.batch_key(b)
    db[key].pop("persistent")
    autotune._store(db)
    m = len(calls)
    autotune.tune_batch(FakeBatch([(160, 256, 256)], nt=[600]))
    assert len(calls) > m
