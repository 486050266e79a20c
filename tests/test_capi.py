"""The C ABI library loads without a GPU and exports every function that
include/pefdtd.h declares (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "pefdtd.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pe_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    from pefdtd import _capi
    L = _capi.lib()
    names = _declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(_capi.exported_symbols()) <= set(names)
    assert L.pe_abi_version() == _capi.ABI_VERSION


def test_ctypes_structs_match_header_fields():
    from pefdtd import _capi
    src = open(HEADER).read()
    for struct, cls in (("PeConfig", _capi.PeConfig), ("PeMedium", _capi.PeMedium),
                        ("PeProbe", _capi.PeProbe), ("PeState", _capi.PeState)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), src, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for part in decl.split(","):
                m = re.search(r"\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*(\[\d+\])?\s*$", part.strip())
                fields.append(m.group(1))
        assert [f[0] for f in cls._fields_] == fields, struct


def test_invalid_arguments_fail_cleanly_without_a_device():
    from pefdtd import _capi
    L = _capi.lib()
    h = C.c_void_p()
    cfg = _capi.PeConfig()
    cfg.nz = cfg.ny = cfg.nx = 4
    cfg.n_coeffs = 7                   # refused before any device work
    md, pr = _capi.PeMedium(), _capi.PeProbe()
    labs = np.zeros(64, np.uint16)
    md.labels_dev = labs.ctypes.data
    md.ctab = md.rho = labs.ctypes.data
    rc = L.pe_solver_create(C.byref(cfg), C.byref(md), C.byref(pr), C.byref(h))
    assert rc == _capi.PE_ERR_INVALID
    assert b"order <= 8" in L.pe_last_error()


def test_trace_entry_points_reject_bad_arguments_without_a_device():
    """pe_trace_*: empty batches, bad offsets, short windows and bad filter
    sizes are refused before any device work (reference: the ValueErrors of
    np.argmax on an empty window and of scipy's filtfilt)."""
    from pefdtd import _capi
    L = _capi.lib()
    x = np.zeros(16, np.float32)
    env = np.zeros(16, np.float64)
    off = np.array([0, 16], np.int64)
    bad_off = np.array([1, 16], np.int64)      # must start at 0
    empty = np.array([0, 0], np.int64)          # an empty trace
    p = lambda a: a.ctypes.data                 # noqa: E731
    assert L.pe_trace_envelope(p(x), _capi.PE_F32, p(off), 0, p(env), None) == _capi.PE_ERR_INVALID
    assert L.pe_trace_envelope(p(x), _capi.PE_F32, p(bad_off), 1, p(env), None) == _capi.PE_ERR_INVALID
    assert L.pe_trace_envelope(p(x), _capi.PE_F32, p(empty), 1, p(env), None) == _capi.PE_ERR_INVALID
    assert L.pe_trace_envelope(p(x), 7, p(off), 1, p(env), None) == _capi.PE_ERR_INVALID
    b = np.ones(3)
    a = np.ones(3)
    zi = np.zeros(2)
    # padlen must be below every trace's length, filters of 2..8 taps
    assert L.pe_trace_detrend(p(x), _capi.PE_F32, p(off), 1, p(b), p(a), 3, p(zi), 16, p(env),
                              None) == _capi.PE_ERR_INVALID
    assert L.pe_trace_detrend(p(x), _capi.PE_F32, p(off), 1, p(b), p(a), 9, p(zi), 9, p(env),
                              None) == _capi.PE_ERR_INVALID
    win = np.array([4, 6], np.int64)            # hi must exceed lo + 2
    dt = np.array([1e-8])
    out = np.zeros(3)
    assert L.pe_trace_pick(p(env), p(off), 1, p(win), p(dt), p(out), None) == _capi.PE_ERR_INVALID
    win4 = np.array([5, 5, 0, 16], np.int64)    # empty E1 window
    tf = np.array([1e-8, 1e8])
    assert L.pe_trace_analyse(p(x), _capi.PE_F32, p(env), p(off), 1, p(win4), p(tf), p(out),
                              None) == _capi.PE_ERR_INVALID
