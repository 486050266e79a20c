"""Schedule autotuner for batched solves.

Picks, by timing the batch itself on its own device, the planes per z-march
(the work-item size: shorter marches give more items and better balance
across the 148 SMs, longer ones spend less on each march's start-up planes),
the number of steps per captured CUDA graph, and the launch mode: one
stress and one velocity launch per step, or one persistent launch per graph
chunk (pefdtd.batch.BatchSolver.set_persistent). The tile shapes are not a
choice: the pair-column kernels' tiles are fixed by their register and
shared-memory budget (two 256-thread blocks per SM). The timed steps advance the
batch's state, which is zeroed afterwards, so tuning leaves a batch exactly
as it found a fresh one. Results are cached per device and batch signature in
a JSON file ($PEFDTD_CACHE or ~/.cache/pefdtd/autotune.json).
"""
from __future__ import annotations

import json
import os

Z_CANDIDATES = (16, 24, 32, 40, 56, 80, 120, 160)
CHUNK_CANDIDATES = (50, 100, 200, 400)


def _cache_path():
    base = os.environ.get("PEFDTD_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "pefdtd")
    return os.path.join(base, "autotune.json")


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(db):
    p = _cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1)
        os.replace(tmp, p)
    except OSError:
        pass


def batch_key(batch):
    torch = batch.torch
    name = torch.cuda.get_device_name(batch.device)
    shapes = sorted(tuple(s) for s in batch.shapes)
    return f"{name}|{batch.npdt.__name__}|{len(shapes)}|" + ";".join("x".join(map(str, s)) for s in shapes)


def time_steps(batch, steps, warmup=2):
    """Mean device milliseconds per step over `steps` steps (CUDA events)."""
    torch = batch.torch
    batch.run(0, warmup)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    batch.run(warmup, warmup + steps)
    end.record()
    end.synchronize()
    batch.check_status()
    return start.elapsed_time(end) / steps


def tune_batch(batch, steps=None, use_cache=True):
    """Choose and apply (z_chunk, chunk_steps); returns them with timings."""
    key = batch_key(batch)
    db = _load() if use_cache else {}
    if use_cache and key in db and "persistent" in db[key]:
        z, c = db[key]["z_chunk"], db[key]["chunk_steps"]
        batch.schedule(z, c)
        batch.set_persistent(db[key]["persistent"])
        return db[key]
    maxnt = min(batch.nt)
    nz_max = max(s[0] for s in batch.shapes)
    steps = steps or max(4, min(12, maxnt - 3))
    trials = {}
    for z in Z_CANDIDATES:
        if z > nz_max and z != Z_CANDIDATES[0]:
            continue
        batch.schedule(z, 1)   # graphs of 1 step: time the kernels, not the graph length
        trials[z] = time_steps(batch, steps)
        batch.reset()
    best_z = min(trials, key=trials.get)
    chunk_trials = {}
    for c in CHUNK_CANDIDATES:
        if c + 2 > maxnt:
            continue
        batch.schedule(best_z, c)
        chunk_trials[c] = time_steps(batch, c)
        batch.reset()
    best_c = min(chunk_trials, key=chunk_trials.get) if chunk_trials else 200
    batch.schedule(best_z, best_c)
    # launch mode at the chosen layout
    mode_trials = {}
    if chunk_trials and batch.set_persistent(True):
        mode_trials["persistent"] = time_steps(batch, best_c)
        batch.reset()
        batch.set_persistent(False)
        mode_trials["per_step"] = chunk_trials[best_c]
    persistent = bool(mode_trials) and mode_trials["persistent"] < mode_trials["per_step"]
    batch.set_persistent(persistent)
    res = dict(z_chunk=best_z, chunk_steps=best_c, persistent=persistent, ms_per_step_by_z=trials,
               ms_per_step_by_chunk=chunk_trials, ms_per_step_by_mode=mode_trials)
    if use_cache:
        db[key] = res
        _store(db)
    return res
