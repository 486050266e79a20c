"""TEST INFRASTRUCTURE ONLY — ctypes front end of the CPU oracle
(oracle/fdtd_oracle.c) and of the reference-kernel harnesses
(oracle/ref_harness.cpp on the host, oracle/ref_gpu_harness.cu on the GPU,
built into oracle/_ref by oracle/build.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module; the product package never does.

Problem dictionaries use the product's inputs:
  mats (nz, ny, nx) int, Ct (n_mat, 36), rho_t (n_mat,), damp (f32 volume
  or None), coeffs, inv_h/dt/dt_h (rounded to the working type by the
  caller, as the reference rounds them: np.float32(1/h), np.float32(dt),
  np.float32(dt/h)), src_idx/src_w, rec_off/rec_idx/rec_w, wavelet, record.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_REC = {"pressure": 0, "vx": 1, "vy": 2, "vz": 3}


class _OracleProblem(C.Structure):
    _fields_ = [("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int), ("n_mat", C.c_int),
                ("nc", C.c_int), ("coeffs", C.c_double * 4), ("inv_h", C.c_double),
                ("dt", C.c_double), ("dt_h", C.c_double), ("record", C.c_int),
                ("damped_record", C.c_int), ("fma_mode", C.c_int), ("nt", C.c_int),
                ("n_threads", C.c_int), ("n_src", C.c_int), ("n_rec_groups", C.c_int),
                ("mats", C.c_void_p), ("ctab", C.c_void_p), ("rho", C.c_void_p),
                ("damp", C.c_void_p), ("src_idx", C.c_void_p), ("src_w", C.c_void_p),
                ("wavelet", C.c_void_p), ("rec_off", C.c_void_p), ("rec_idx", C.c_void_p),
                ("rec_w", C.c_void_p)]


_oracle = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p).value


def oracle_lib():
    global _oracle
    if _oracle is None:
        path = _build.build_oracle()
        L = C.CDLL(path)
        L.oracle_problem_size.restype = C.c_int
        if L.oracle_problem_size() != C.sizeof(_OracleProblem):
            raise RuntimeError("oracle ABI mismatch")
        L.oracle_forward_f32.argtypes = [C.POINTER(_OracleProblem), C.c_void_p, C.c_void_p]
        L.oracle_forward_f64.argtypes = [C.POINTER(_OracleProblem), C.c_void_p, C.c_void_p]
        _oracle = L
    return _oracle


def ref_lib():
    """The reference-kernel harness, or None where it cannot be built."""
    global _ref
    if _ref is None:
        path = _build.build_ref()
        if path is None or not os.path.exists(path):
            return None
        L = C.CDLL(path)
        i64p = C.c_void_p
        L.ref_labels_forward.argtypes = (
            [C.c_int] * 3 + [C.c_void_p] * 6 + [C.c_int, C.c_float, C.c_float, C.c_float, C.c_int,
                                                i64p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                C.c_int, i64p, i64p, C.c_void_p, C.c_int,
                                                C.c_void_p, C.c_void_p, C.c_int])
        L.ref_dense_forward.argtypes = (
            [C.c_int] * 3 + [C.c_void_p] * 7 + [C.c_int, C.c_float, C.c_float, C.c_float,
                                                i64p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                C.c_int, i64p, i64p, C.c_void_p, C.c_int,
                                                C.c_void_p, C.c_void_p, C.c_int])
        _ref = L
    return _ref


_ref_gpu = None


def ref_gpu_lib():
    """The reference kernels built for the GPU (oracle/_ref/libref_gpu.so),
    or None where they cannot be built or loaded."""
    global _ref_gpu
    if _ref_gpu is None:
        path = _build.build_ref_gpu()
        if path is None or not os.path.exists(path):
            return None
        L = C.CDLL(path)
        i64p = C.c_void_p
        L.refgpu_labels_forward.argtypes = (
            [C.c_int] * 3 + [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                                C.c_float, C.c_float, C.c_int, i64p, C.c_void_p, C.c_int,
                                                C.c_void_p, C.c_int, C.c_int, i64p, i64p, C.c_void_p,
                                                C.c_int, C.c_void_p])
        L.refgpu_dense_forward.argtypes = (
            [C.c_int] * 3 + [C.c_void_p] * 7 + [C.c_int, C.c_float, C.c_float, C.c_float, i64p,
                                                C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, i64p,
                                                i64p, C.c_void_p, C.c_int, C.c_void_p])
        _ref_gpu = L
    return _ref_gpu


def _probe_arrays(prob):
    return (np.ascontiguousarray(prob["src_idx"], np.int64), np.ascontiguousarray(prob["src_w"], np.float32),
            np.ascontiguousarray(prob["wavelet"], np.float32), np.ascontiguousarray(prob["rec_off"], np.int64),
            np.ascontiguousarray(prob["rec_idx"], np.int64), np.ascontiguousarray(prob["rec_w"], np.float32))


def run_reference_labels_gpu(prob, slab=32):
    """The reference's own label-path kernels (strains_zp, stress_lab_u,
    vel_zp) on the GPU, nvcc-built with default FMA contraction, launched as
    sim/core/fdtd.py:1741-1816 launches them. Needs uint8-range materials."""
    L = ref_gpu_lib()
    if L is None:
        raise RuntimeError("GPU reference harness unavailable (oracle/_ref not built)")
    mats = np.asarray(prob["mats"])
    if mats.max() > 255:
        raise ValueError("the reference label path holds materials in uint8")
    mats = np.ascontiguousarray(mats, np.uint8)
    nz, ny, nx = mats.shape
    Ct = np.ascontiguousarray(prob["Ct"], np.float32).reshape(-1, 36)
    act = np.ascontiguousarray((np.abs(Ct) > 0).any(axis=0).astype(np.int32))
    rho = np.ascontiguousarray(prob["rho_t"], np.float32)
    damp = prob.get("damp")
    damp = np.ascontiguousarray(damp, np.float32) if damp is not None else None
    coeffs = np.ascontiguousarray(prob["coeffs"], np.float32)
    s_idx, s_w, wav, r_off, r_idx, r_w = _probe_arrays(prob)
    nt = int(prob["nt"])
    ng = len(r_off) - 1
    out = np.zeros((nt, ng), np.float32)
    rc = L.refgpu_labels_forward(nz, ny, nx, _p(mats), _p(Ct), _p(act), _p(rho), len(rho), _p(damp),
                                 _p(coeffs), len(coeffs), float(np.float32(prob["inv_h"])),
                                 float(np.float32(prob["dt"])), float(np.float32(prob["dt_h"])), slab,
                                 _p(s_idx), _p(s_w), len(s_idx), _p(wav), nt, ng, _p(r_off), _p(r_idx),
                                 _p(r_w), _REC[prob.get("record", "pressure")], _p(out))
    if rc:
        raise RuntimeError(f"GPU reference harness failed with code {rc}")
    return out


def run_reference_dense_gpu(prob):
    """The reference's dense kernels (strains, stress_acc, vel_update) with
    end-of-step damping on the GPU, nvcc-built with default FMA contraction,
    launched as sim/core/fdtd.py:875-921 launches them; any number of
    materials (36 per-cell stiffness planes)."""
    L = ref_gpu_lib()
    if L is None:
        raise RuntimeError("GPU reference harness unavailable (oracle/_ref not built)")
    mats = np.asarray(prob["mats"]).astype(np.int64)
    nz, ny, nx = mats.shape
    Ct = np.asarray(prob["Ct"], np.float32).reshape(-1, 36)
    Cflat = np.ascontiguousarray(np.moveaxis(Ct[mats], -1, 0))
    act = np.ascontiguousarray((np.abs(Ct) > 0).any(axis=0).astype(np.int32))
    rho_cell = np.asarray(prob["rho_t"], np.float32)[mats].astype(float)
    rv = [np.ascontiguousarray(_face_density(rho_cell, ax), np.float32) for ax in (2, 1, 0)]
    damp = prob.get("damp")
    damp = np.ascontiguousarray(damp, np.float32) if damp is not None else None
    coeffs = np.ascontiguousarray(prob["coeffs"], np.float32)
    s_idx, s_w, wav, r_off, r_idx, r_w = _probe_arrays(prob)
    nt = int(prob["nt"])
    ng = len(r_off) - 1
    out = np.zeros((nt, ng), np.float32)
    rc = L.refgpu_dense_forward(nz, ny, nx, _p(Cflat), _p(act), _p(rv[0]), _p(rv[1]), _p(rv[2]), _p(damp),
                                _p(coeffs), len(coeffs), float(np.float32(prob["inv_h"])),
                                float(np.float32(prob["dt"])), float(np.float32(prob["dt_h"])), _p(s_idx),
                                _p(s_w), len(s_idx), _p(wav), nt, ng, _p(r_off), _p(r_idx), _p(r_w),
                                _REC[prob.get("record", "pressure")], _p(out))
    if rc:
        raise RuntimeError(f"GPU reference harness failed with code {rc}")
    return out


def run_oracle(prob, dtype=np.float32, fma_mode=1, n_threads=0, return_state=False):
    """Traces (nt, n_groups) of the C oracle in dtype (float32 or float64)."""
    dt_ = np.dtype(dtype)
    L = oracle_lib()
    mats = np.ascontiguousarray(prob["mats"], np.int32)
    nz, ny, nx = mats.shape
    Ct = np.ascontiguousarray(prob["Ct"], dt_).reshape(-1, 36)
    rho = np.ascontiguousarray(prob["rho_t"], dt_)
    damp = prob.get("damp")
    damp = np.ascontiguousarray(damp, np.float32) if damp is not None else None
    src_idx = np.ascontiguousarray(prob["src_idx"], np.int64)
    src_w = np.ascontiguousarray(prob["src_w"], dt_)
    wav = np.ascontiguousarray(prob["wavelet"], dt_)
    rec_off = np.ascontiguousarray(prob["rec_off"], np.int64)
    rec_idx = np.ascontiguousarray(prob["rec_idx"], np.int64)
    rec_w = np.ascontiguousarray(prob["rec_w"], dt_)
    nt = int(prob["nt"])
    coeffs = np.asarray(prob["coeffs"], float)
    P = _OracleProblem()
    P.nz, P.ny, P.nx = nz, ny, nx
    P.n_mat = len(rho)
    P.nc = len(coeffs)
    for j in range(len(coeffs)):
        P.coeffs[j] = float(dt_.type(coeffs[j]))
    P.inv_h = float(dt_.type(prob["inv_h"]))
    P.dt = float(dt_.type(prob["dt"]))
    P.dt_h = float(dt_.type(prob["dt_h"]))
    P.record = _REC[prob.get("record", "pressure")]
    P.damped_record = int(bool(prob.get("damped_record", False)))
    P.fma_mode = int(fma_mode)
    P.nt = nt
    P.n_threads = int(n_threads)
    P.n_src = len(src_idx)
    P.n_rec_groups = len(rec_off) - 1
    P.mats, P.ctab, P.rho, P.damp = _p(mats), _p(Ct), _p(rho), _p(damp)
    P.src_idx, P.src_w, P.wavelet = _p(src_idx), _p(src_w), _p(wav)
    P.rec_off, P.rec_idx, P.rec_w = _p(rec_off), _p(rec_idx), _p(rec_w)
    out = np.zeros((nt, P.n_rec_groups), dt_)
    state = np.zeros((9, nz, ny, nx), dt_) if return_state else None
    fn = L.oracle_forward_f64 if dt_ == np.float64 else L.oracle_forward_f32
    rc = fn(C.byref(P), _p(out), _p(state))
    if rc:
        raise RuntimeError(f"oracle failed with code {rc}")
    return (out, state) if return_state else out


def run_reference_labels(prob, slab=32, n_threads=0, return_state=False):
    """The reference's own label-path kernels (strains_zp, stress_lab_u,
    vel_zp) run on the host. Needs uint8-range materials (< 256)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference harness unavailable (oracle/_ref not built)")
    mats = np.asarray(prob["mats"])
    if mats.max() > 255:
        raise ValueError("the reference label path holds materials in uint8")
    mats = np.ascontiguousarray(mats, np.uint8)
    nz, ny, nx = mats.shape
    Ct = np.ascontiguousarray(prob["Ct"], np.float32).reshape(-1, 36)
    act = np.ascontiguousarray((np.abs(Ct) > 0).any(axis=0).astype(np.int32))
    rho = np.ascontiguousarray(prob["rho_t"], np.float32)
    damp = prob.get("damp")
    damp = np.ascontiguousarray(damp, np.float32) if damp is not None else None
    coeffs = np.ascontiguousarray(prob["coeffs"], np.float32)
    src_idx = np.ascontiguousarray(prob["src_idx"], np.int64)
    src_w = np.ascontiguousarray(prob["src_w"], np.float32)
    wav = np.ascontiguousarray(prob["wavelet"], np.float32)
    rec_off = np.ascontiguousarray(prob["rec_off"], np.int64)
    rec_idx = np.ascontiguousarray(prob["rec_idx"], np.int64)
    rec_w = np.ascontiguousarray(prob["rec_w"], np.float32)
    nt = int(prob["nt"])
    ng = len(rec_off) - 1
    out = np.zeros((nt, ng), np.float32)
    state = np.zeros((9, nz, ny, nx), np.float32) if return_state else None
    rc = L.ref_labels_forward(nz, ny, nx, _p(mats), _p(Ct), _p(act), _p(rho), _p(damp),
                              _p(coeffs), len(coeffs), float(np.float32(prob["inv_h"])),
                              float(np.float32(prob["dt"])), float(np.float32(prob["dt_h"])),
                              slab, _p(src_idx), _p(src_w), len(src_idx), _p(wav), nt, ng,
                              _p(rec_off), _p(rec_idx), _p(rec_w), _REC[prob.get("record", "pressure")],
                              _p(out), _p(state), int(n_threads))
    if rc:
        raise RuntimeError(f"reference harness failed with code {rc}")
    return (out, state) if return_state else out


def run_reference_dense(prob, n_threads=0, return_state=False):
    """The reference's dense kernels (strains, stress_acc, vel_update) with
    end-of-step damping, on the host; any number of materials."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference harness unavailable (oracle/_ref not built)")
    mats = np.asarray(prob["mats"]).astype(np.int64)
    nz, ny, nx = mats.shape
    Ct = np.asarray(prob["Ct"], np.float32).reshape(-1, 36)
    Cflat = np.ascontiguousarray(np.moveaxis(Ct[mats], -1, 0))
    act = np.ascontiguousarray((np.abs(Ct) > 0).any(axis=0).astype(np.int32))
    rho_cell = np.asarray(prob["rho_t"], np.float32)[mats].astype(float)
    rv = [np.ascontiguousarray(_face_density(rho_cell, ax), np.float32) for ax in (2, 1, 0)]
    damp = prob.get("damp")
    damp = np.ascontiguousarray(damp, np.float32) if damp is not None else None
    coeffs = np.ascontiguousarray(prob["coeffs"], np.float32)
    src_idx = np.ascontiguousarray(prob["src_idx"], np.int64)
    src_w = np.ascontiguousarray(prob["src_w"], np.float32)
    wav = np.ascontiguousarray(prob["wavelet"], np.float32)
    rec_off = np.ascontiguousarray(prob["rec_off"], np.int64)
    rec_idx = np.ascontiguousarray(prob["rec_idx"], np.int64)
    rec_w = np.ascontiguousarray(prob["rec_w"], np.float32)
    nt = int(prob["nt"])
    ng = len(rec_off) - 1
    out = np.zeros((nt, ng), np.float32)
    state = np.zeros((9, nz, ny, nx), np.float32) if return_state else None
    rc = L.ref_dense_forward(nz, ny, nx, _p(Cflat), _p(act), _p(rv[0]), _p(rv[1]), _p(rv[2]),
                             _p(damp), _p(coeffs), len(coeffs), float(np.float32(prob["inv_h"])),
                             float(np.float32(prob["dt"])), float(np.float32(prob["dt_h"])),
                             _p(src_idx), _p(src_w), len(src_idx), _p(wav), nt, ng, _p(rec_off),
                             _p(rec_idx), _p(rec_w), _REC[prob.get("record", "pressure")],
                             _p(out), _p(state), int(n_threads))
    if rc:
        raise RuntimeError(f"reference harness failed with code {rc}")
    return (out, state) if return_state else out


def _face_density(rho, ax):
    m = np.empty_like(rho)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[ax] = slice(0, -1)
    hi[ax] = slice(1, None)
    m[tuple(lo)] = 0.5 * (rho[tuple(lo)] + rho[tuple(hi)])
    last = [slice(None)] * 3
    last[ax] = slice(-1, None)
    m[tuple(last)] = rho[tuple(last)]
    return m


def problem_from_workload(p, record=None, damped_record=True, use_sponge=True, damp_mask=None,
                          dtype=np.float32, Ct=None, rho_t=None):
    """Oracle/harness problem dict from a workload dict (pefdtd.workloads):
    the combined f32 damping volume the reference multiplies together
    (sponge_profile * damp_mask), flat probe lists in caller order, and the
    scalars rounded to the working type as the reference rounds them."""
    from pefdtd import damping
    from pefdtd.fdtd import _flat_probe
    shape = p["lab"].shape
    damp = None
    if use_sponge and p["sponge"] > 0:
        damp = damping.sponge_profile(shape, p["sponge"])
    if damp_mask is not None:
        damp = damp_mask if damp is None else (damp * damp_mask).astype(np.float32)
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, p["src_pts"], p["rec_groups"], dtype)
    h, dt = p["h"], p["dt"]
    cast = np.dtype(dtype).type
    return dict(mats=np.asarray(p["mats"]).astype(np.int32), Ct=p["Ct"] if Ct is None else Ct,
                rho_t=p["rho_t"] if rho_t is None else rho_t, damp=damp,
                coeffs=np.asarray(p["coeffs"], dtype), inv_h=cast(1.0 / h), dt=cast(dt),
                dt_h=cast(dt / h), src_idx=s_idx, src_w=s_w, rec_off=r_off, rec_idx=r_idx,
                rec_w=r_w, wavelet=np.asarray(p["wavelet"], dtype)[:p["nt"]], nt=p["nt"],
                record=record or p["record"], damped_record=damped_record)
