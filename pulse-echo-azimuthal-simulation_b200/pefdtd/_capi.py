"""ctypes binding of include/pefdtd.h (the library built by pefdtd/build.py).

Loading never falls back to anything: if the CUDA library is missing or was
built for another ABI, import of the solver entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

PE_OK, PE_ERR_INVALID, PE_ERR_CUDA, PE_ERR_NOMEM, PE_ERR_UNSUPPORTED, PE_ERR_TIMEOUT = range(6)
PE_F32, PE_F64 = 0, 1
REC_KIND = {"pressure": 0, "vx": 1, "vy": 2, "vz": 3}
ABI_VERSION = 1
MAX_MATERIALS = 16383


class PeConfig(C.Structure):
    _fields_ = [("nz", C.c_int32), ("ny", C.c_int32), ("nx", C.c_int32),
                ("dtype", C.c_int32), ("n_coeffs", C.c_int32),
                ("coeffs", C.c_double * 4), ("h", C.c_double), ("dt", C.c_double),
                ("record", C.c_int32), ("damped_record", C.c_int32),
                ("n_mat", C.c_int32), ("chunk_steps", C.c_int32),
                ("tile_x", C.c_int32), ("tile_y", C.c_int32), ("z_chunk", C.c_int32),
                ("variant", C.c_int32)]


KERNEL_VARIANT = {"tiled": 0, "simple": 1, "column": 2, "dense": 3}


class PeMedium(C.Structure):
    _fields_ = [("labels_dev", C.c_void_p), ("damp_volume_dev", C.c_void_p),
                ("ctab", C.c_void_p), ("rho", C.c_void_p),
                ("sponge_z", C.c_void_p), ("sponge_y", C.c_void_p), ("sponge_x", C.c_void_p)]


class PeProbe(C.Structure):
    _fields_ = [("n_src", C.c_int32), ("src_idx", C.c_void_p), ("src_w", C.c_void_p),
                ("n_groups", C.c_int32), ("rec_off", C.c_void_p), ("rec_idx", C.c_void_p),
                ("rec_w", C.c_void_p)]


class PeState(C.Structure):
    _fields_ = [("v", C.c_void_p * 3), ("s", C.c_void_p * 6)]


class PeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pefdtd error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded CUDA library (built on first use if stale)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if _build.is_stale():
            path = _build.build()
        if not os.path.exists(path):
            raise RuntimeError(f"pefdtd CUDA library missing at {path}")
        L = C.CDLL(path)
        L.pe_abi_version.restype = C.c_int
        L.pe_last_error.restype = C.c_char_p
        L.pe_solver_create.argtypes = [C.POINTER(PeConfig), C.POINTER(PeMedium),
                                       C.POINTER(PeProbe), C.POINTER(C.c_void_p)]
        L.pe_solver_set_wavelet.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.pe_solver_run.argtypes = [C.c_void_p, C.POINTER(PeState), C.c_void_p, C.c_int64,
                                    C.c_int64, C.c_void_p]
        L.pe_solver_launch_count.argtypes = [C.c_void_p]
        L.pe_solver_launch_count.restype = C.c_int64
        L.pe_solver_destroy.argtypes = [C.c_void_p]
        L.pe_solver_status.argtypes = [C.c_void_p]
        L.pe_solver_profile.argtypes = [C.c_void_p, C.POINTER(PeState), C.c_int,
                                        C.POINTER(C.c_float), C.c_void_p]
        L.pe_forward_host.argtypes = [C.POINTER(PeConfig), C.c_void_p, C.c_void_p,
                                      C.POINTER(PeMedium), C.POINTER(PeProbe), C.c_void_p,
                                      C.c_int64, C.c_void_p]
        L.pe_batch_create.argtypes = [C.c_int, C.POINTER(PeConfig), C.POINTER(PeMedium),
                                      C.POINTER(PeProbe), C.POINTER(C.c_void_p)]
        L.pe_batch_schedule.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.pe_batch_set_persistent.argtypes = [C.c_void_p, C.c_int]
        L.pe_batch_set_wavelet.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        L.pe_batch_run.argtypes = [C.c_void_p, C.POINTER(PeState), C.POINTER(C.c_void_p),
                                   C.c_int64, C.c_int64, C.c_void_p]
        L.pe_batch_status.argtypes = [C.c_void_p]
        L.pe_batch_launch_count.argtypes = [C.c_void_p]
        L.pe_batch_launch_count.restype = C.c_int64
        L.pe_batch_destroy.argtypes = [C.c_void_p]
        L.pe_label_cylinder.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_void_p]
        L.pe_rotated_grid.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                      C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        L.pe_trace_envelope.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                        C.c_void_p]
        L.pe_trace_detrend.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                       C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                       C.c_void_p]
        L.pe_trace_pick.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
        L.pe_trace_analyse.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        if L.pe_abi_version() != ABI_VERSION:
            raise RuntimeError("pefdtd library ABI mismatch; rebuild with pefdtd.build")
        _lib = L
    return _lib


def check(rc):
    """Raise the reference's error class for a failed call."""
    if rc == PE_OK:
        return
    msg = lib().pe_last_error().decode(errors="replace")
    if rc == PE_ERR_INVALID:
        raise ValueError(msg)
    raise PeError(rc, msg)


def ptr(a):
    """Host address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array handed to the C ABI must be C-contiguous")
    return a.ctypes.data_as(C.c_void_p).value


def exported_symbols():
    return ["pe_abi_version", "pe_last_error", "pe_solver_create", "pe_solver_set_wavelet",
            "pe_solver_run", "pe_solver_launch_count", "pe_solver_profile", "pe_solver_status",
            "pe_solver_destroy",
            "pe_forward_host", "pe_release_cached_memory", "pe_label_cylinder", "pe_rotated_grid", "pe_batch_create", "pe_batch_schedule", "pe_batch_set_persistent",
            "pe_batch_set_wavelet", "pe_batch_run", "pe_batch_status", "pe_batch_launch_count",
            "pe_batch_destroy", "pe_trace_envelope", "pe_trace_detrend", "pe_trace_pick",
            "pe_trace_analyse"]
