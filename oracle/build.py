"""TEST INFRASTRUCTURE ONLY — build recipe for the CPU oracle and the
reference-kernel harness.

* ``oracle/_build/liboracle.so``  from oracle/fdtd_oracle.c (the C restatement).
* ``oracle/_ref/libref_gpu.so``   the same kernel strings behind
  oracle/ref_gpu_harness.cu, compiled by nvcc for the GPU (default FMA
  contraction, as the reference's NVRTC build).
* ``oracle/_ref/libref_cpu.so``   from oracle/ref_harness.cpp plus the
  reference's own CUDA-C kernel strings, read from the reference module where
  it lies (``sim/core/fdtd.py`` of Jerome-Graves/pulse-echo-azimuthal-simulation)
  and written to ``oracle/_ref/ref_kernels.inc``. Only possible where the
  reference tree is present; elsewhere the prebuilt library is used.

Both outputs are git-ignored. Flags: no fast-math and no FP contraction, so
every product and sum is rounded as written; no ``-march=native`` so the
library runs on any x86-64 host it is copied to.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")


def _reference_root():
    """The reference checkout to read the kernel strings from
    (PE_REFERENCE_ROOT): required to build oracle/_ref, no default; without
    it the prebuilt library is used."""
    return os.environ.get("PE_REFERENCE_ROOT")


ORACLE_LIB = os.path.join(BUILD, "liboracle.so")
REF_CPU_LIB = os.path.join(REF_OUT, "libref_cpu.so")

_CFLAGS = ["-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-Wall",
           "-Wno-unused-function"]


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force=False):
    srcs = [os.path.join(HERE, "fdtd_oracle.c"), os.path.join(HERE, "fdtd_oracle_impl.h")]
    if not force and _newer(ORACLE_LIB, srcs):
        return ORACLE_LIB
    os.makedirs(BUILD, exist_ok=True)
    tmp = ORACLE_LIB + ".tmp"
    subprocess.check_call(["gcc", *_CFLAGS, "-o", tmp, srcs[0], "-lm"])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def _reference_kernel_sources(root):
    """The reference's own kernel source strings, unmodified, from the module."""
    sys.path.insert(0, os.path.join(root, "sim", "core"))
    sys.path.insert(0, os.path.join(root, "vendor"))
    try:
        import importlib
        fd = importlib.import_module("fdtd")
        parts = [
            ("strains_zp (sim/core/fdtd.py:1102-1177)", fd._STRAIN_ZP_SRC),
            ("stress_lab_u (sim/core/fdtd.py:594-689)", fd._stress_unrolled_src()),
            ("vel_zp (sim/core/fdtd.py:1179-1257)", fd._VEL_ZP_SRC),
            ("strains (sim/core/fdtd.py:463-505)", fd._STRAIN_SRC),
            ("stress_acc (sim/core/fdtd.py:507-583)", fd._STRESS_SRC),
            ("vel_update (sim/core/fdtd.py:392-442)", fd._VEL_SRC),
        ]
    finally:
        sys.path.pop(0)
        sys.path.pop(0)
    out = ["// GENERATED by oracle/build.py from the reference module; do not commit.\n"]
    for name, src in parts:
        out.append(f"\n// ---- {name}\n")
        out.append(src)
    return "".join(out)


def build_ref(force=False):
    """Build oracle/_ref/libref_cpu.so; returns its path or None if impossible."""
    harness = os.path.join(HERE, "ref_harness.cpp")
    REFERENCE_ROOT = _reference_root()
    if not REFERENCE_ROOT:
        if not os.path.exists(REF_CPU_LIB):
            print("oracle/build.py: PE_REFERENCE_ROOT is not set, so oracle/_ref (the reference's "
                  "own kernels built for the host) cannot be built; set it to the reference "
                  "checkout to build it", file=sys.stderr)
            return None
        return REF_CPU_LIB
    core = os.path.join(REFERENCE_ROOT, "sim", "core", "fdtd.py")
    if not os.path.exists(core):
        raise FileNotFoundError(f"PE_REFERENCE_ROOT={REFERENCE_ROOT!r} holds no sim/core/fdtd.py")
    if not force and _newer(REF_CPU_LIB, [core, harness, __file__]):
        return REF_CPU_LIB
    os.makedirs(REF_OUT, exist_ok=True)
    inc = os.path.join(REF_OUT, "ref_kernels.inc")
    with open(inc, "w") as f:
        f.write(_reference_kernel_sources(REFERENCE_ROOT))
    tmp = REF_CPU_LIB + ".tmp"
    subprocess.check_call(["g++", "-std=c++17", *_CFLAGS, "-Wno-unused-variable",
                           "-I", HERE, "-o", tmp, harness])
    os.replace(tmp, REF_CPU_LIB)
    return REF_CPU_LIB


REF_GPU_LIB = os.path.join(REF_OUT, "libref_gpu.so")


def build_ref_gpu(force=False):
    """Build oracle/_ref/libref_gpu.so: the reference's kernel strings
    (oracle/_ref/ref_kernels.inc, written by build_ref) behind the GPU driver
    restatement oracle/ref_gpu_harness.cu, compiled by nvcc for sm_100a with
    its default FMA contraction (as NVRTC compiles them for the reference).
    Returns its path, or None where it cannot be built."""
    harness = os.path.join(HERE, "ref_gpu_harness.cu")
    inc = os.path.join(REF_OUT, "ref_kernels.inc")
    if not os.path.exists(inc):
        return REF_GPU_LIB if os.path.exists(REF_GPU_LIB) else None
    if not force and _newer(REF_GPU_LIB, [inc, harness]):
        return REF_GPU_LIB
    nvcc = None
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            nvcc = c
            break
    if nvcc is None:
        import shutil
        nvcc = shutil.which("nvcc")
    if nvcc is None:
        return REF_GPU_LIB if os.path.exists(REF_GPU_LIB) else None
    tmp = REF_GPU_LIB + ".tmp"
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                           "-Xcompiler", "-fPIC", "-shared", "-I", HERE, "-o", tmp, harness])
    os.replace(tmp, REF_GPU_LIB)
    return REF_GPU_LIB


def build_all(force=False):
    return build_oracle(force), build_ref(force), build_ref_gpu(force)


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
