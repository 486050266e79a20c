"""The batched sweep driver's protocol against the reference sweep engine
(tests/golden/sweep_protocol.npz): visiting order, per-azimuth solver
arguments, az{ddd}.npz contents, status.json, STOP and resume. The solver
is a stand-in returning a fixed synthetic trace, as in the fixture; the GPU
solve itself is covered in test_sweep_gpu.py."""
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import synthetic_echo

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CFG = dict(f0_mhz=0.5, ppw=6.0, az_start=0, az_stop=360, az_step=45, diameter_mm=80.0,
           thickness_mm=10.0, n_grains=12, sponge=10, seed=5)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def gold():
    with np.load(os.path.join(GOLD, "sweep_protocol.npz")) as z:
        return {k: z[k] for k in z.files}


def _stub(seen):
    def solve(setups, progress):
        out = []
        for s in setups:
            seen.append(s)
            out.append(synthetic_echo(s["nt"], s["dt"], s["f0"]).astype(float))
        progress(1.0)
        return out
    return solve


def test_visiting_orders(gold):
    from pefdtd import sweep
    for n in range(70):
        assert sweep.bit_reversed_order(n) == list(gold[f"bitrev_{n}"])
    for start, stop, step, mode in ((0, 360, 1, "progressive"), (10, 350, 7, "progressive"),
                                    (0, 180, 4, "progressive"), (0, 360, 5, "sequential")):
        c = dict(az_start=start, az_stop=stop, az_step=step, sweep_order=mode)
        assert sweep.azimuths(c) == list(gold[f"az_{start}_{stop}_{step}_{mode}"])


def test_setups_and_files_match_reference(tmp_path, gold):
    from pefdtd import sweep
    sweep.create("fx", str(tmp_path), **CFG)
    cfg = sweep.load("fx", str(tmp_path))
    seen = []
    assert sweep.run(cfg, labeller="exact", solver=_stub(seen), batch=3, log=lambda *a: None) == "complete"
    assert [s["az"] for s in seen] == list(gold["order"])
    for s in seen:
        az, sp = s["az"], s["spec"]
        lab = sp["mats"].astype(np.int32) - 1
        assert tuple(lab.shape) == tuple(gold[f"{az}_lab_shape"])
        assert _sha(lab) == str(gold[f"{az}_lab_sha"]), az
        assert _sha(np.asarray(sp["damp_volume"], np.float32)) == str(gold[f"{az}_dm_sha"])
        assert _sha(np.asarray(sp["wavelet"], np.float64)) == str(gold[f"{az}_wav_sha"])
        assert np.array_equal(s["axes"], gold[f"{az}_axes"])
        assert s["dt"] == float(gold[f"{az}_dt"]) and s["nt"] == int(gold[f"{az}_nt"])
        src = np.stack(np.unravel_index(sp["src_idx"], lab.shape), 1)
        assert np.array_equal(src, gold[f"{az}_src"])
        assert np.all(sp["src_w"] == float(gold[f"{az}_w"]))
        assert np.array_equal(sp["coeffs"], gold[f"{az}_coeffs"])
        with np.load(os.path.join(tmp_path, "fx", f"az{az:03d}.npz")) as z:
            keys = sorted(k[len(f"{az}_file_"):] for k in gold if k.startswith(f"{az}_file_"))
            assert sorted(z.files) == keys
            for k in keys:
                g = gold[f"{az}_file_{k}"]
                assert z[k].dtype == g.dtype, k
                assert np.array_equal(z[k], g, equal_nan=True), k
    with open(os.path.join(tmp_path, "fx", "status.json")) as f:
        st = json.load(f)
    assert st["phase"] == str(gold["final_phase"]) and st["done"] == st["total"] == 8


def test_stop_mid_batch_then_resume(tmp_path):
    from pefdtd import sweep
    sweep.create("s", str(tmp_path), **CFG)
    cfg = sweep.load("s", str(tmp_path))
    d = os.path.join(tmp_path, "s")
    open(os.path.join(d, "STOP"), "w").close()        # a stale flag is cleared on start
    calls = []

    def stopping(setups, progress):
        calls.append([s["az"] for s in setups])
        if len(calls) == 2:
            open(os.path.join(d, "STOP"), "w").close()
        progress(0.5)
        return [synthetic_echo(s["nt"], s["dt"], s["f0"]) for s in setups]
    assert sweep.run(cfg, labeller="exact", solver=stopping, batch=3, log=lambda *a: None) == "stopped"
    assert len(calls) == 2
    assert sweep.done_azimuths(cfg) == sorted(calls[0])
    assert not [f for f in os.listdir(d) if ".tmp" in f]
    with open(os.path.join(d, "status.json")) as f:
        assert json.load(f)["phase"] == "stopped"
    seen = []
    assert sweep.run(cfg, labeller="exact", solver=_stub(seen), batch=4, log=lambda *a: None) == "complete"
    assert [s["az"] for s in seen] == [a for a in sweep.azimuths(cfg) if a not in calls[0]]
    assert len(sweep.done_azimuths(cfg)) == 8
    with open(os.path.join(d, "status.json")) as f:
        st = json.load(f)
    assert st["phase"] == "complete" and st["sec_per_az"] is not None
    seen.clear()
    assert sweep.run(cfg, labeller="exact", solver=_stub(seen), log=lambda *a: None) == "complete"
    assert seen == []


def test_legacy_convention_guard_and_no_cuda(tmp_path):
    from pefdtd import sweep
    sweep.create("old", str(tmp_path), **CFG)
    cfg = sweep.load("old", str(tmp_path))
    cfg.pop("axes_convention")
    d = os.path.join(tmp_path, "old")
    np.savez(os.path.join(d, "az000.npz"), trace=np.zeros(3, np.float32))
    assert sweep.run(cfg, labeller="exact", solver=_stub([]), log=lambda *a: None) == "legacy"
    with open(os.path.join(d, "status.json")) as f:
        assert json.load(f)["phase"].startswith("LEGACY")
    import torch
    if not torch.cuda.is_available():
        sweep.create("nc", str(tmp_path), **CFG)
        assert sweep.run(sweep.load("nc", str(tmp_path)), log=lambda *a: None) == "no-cuda"
        with open(os.path.join(tmp_path, "nc", "status.json")) as f:
            assert json.load(f)["phase"] == "NO CUDA - cannot run"
