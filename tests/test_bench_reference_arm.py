"""bench.py's reference arm on the CPU: `--impl reference` times the
reference's own update kernels on the host (oracle/_ref, else the C port)
and prints one JSON line with the bench contract's keys; it loads no library
of the CUDA path."""
import json
import os
import subprocess
import sys

import helpers


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    bench = os.path.join(helpers.ROOT, "bench.py")
    argv = [bench, "--impl", "reference", "--workload", "disk_small", "--steps", "2", "--warmup", "3"]
    # run bench.py as __main__, then report whether this process mapped the
    # CUDA path's library
    probe = ("import runpy, sys; sys.argv = %r; runpy.run_path(%r, run_name='__main__'); "
             "maps = open('/proc/self/maps').read(); "
             "print('CUDA-LIB-LOADED' if 'libpefdtd' in maps else 'CUDA-LIB-ABSENT', file=sys.stderr)" % (argv, bench))
    cmd = [sys.executable, "-c", probe]
    out = subprocess.run(cmd, cwd=helpers.ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "Gcell-updates/s" and d["unit"] == "Gcell-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"] == "disk_small" and d["config"]["grid"] == [64, 96, 96]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port") and cb["cpu_model"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "CUDA-LIB-ABSENT" in out.stderr, out.stderr[-500:]
