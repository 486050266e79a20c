"""The allocation-free labeller entry point (pe_label_cylinder_noalloc).

It serves callers that may not allocate device memory (a framework owns the
device pool, or a pipeline stage must not pay cudaMalloc's implicit
synchronisation): its staging buffer is a fixed file-scope device array. This
checks, through the C ABI, that two calls in a row give exactly the labels of
the allocating entry point pe_label_cylinder, and that oversized requests are
refused. Collected last, so a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from pefdtd import _capi
    L = _capi.lib()
    args = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double,
            C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.pe_label_cylinder_noalloc.argtypes = args
    L.pe_label_cylinder_noalloc_error.restype = C.c_char_p
    return L, _capi


def _call(fn, capi, x, y, z, R, seeds, w, out):
    import torch
    return fn(capi.ptr(x), len(x), capi.ptr(y), len(y), capi.ptr(z), len(z), float(R) ** 2,
              capi.ptr(seeds), capi.ptr(w) if w is not None else None, len(seeds), out.data_ptr(),
              C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_allocating_entry_twice():
    import torch
    from pefdtd import specimen
    L, capi = _lib()
    rng = np.random.default_rng(17)
    cases = [
        (np.ascontiguousarray((np.arange(48) - 23.5) * 0.2e-3), 40, 18, 5e-3, 90, True),
        (np.ascontiguousarray((np.arange(33) - 16.0) * 0.25e-3), 37, 11, 4e-3, 31, False),
    ]
    for xs, ny, nz, R, ns, weighted in cases:
        ys = np.ascontiguousarray(xs[:ny] if ny <= len(xs) else (np.arange(ny) - ny / 2) * 0.2e-3)
        zs = np.ascontiguousarray((np.arange(nz) - (nz - 1) / 2) * 0.2e-3)
        seeds = np.ascontiguousarray(specimen.seed_points(R, nz * 0.2e-3, ns, rng))
        w = np.ascontiguousarray(rng.uniform(0, 3e-7, ns)) if weighted else None
        ref = torch.full((len(zs), len(ys), len(xs)), -7, dtype=torch.int32, device="cuda")
        got = torch.full_like(ref, -9)
        capi.check(_call(L.pe_label_cylinder, capi, xs, ys, zs, R, seeds, w, ref))
        rc = _call(L.pe_label_cylinder_noalloc, capi, xs, ys, zs, R, seeds, w, got)
        assert rc == 0, L.pe_label_cylinder_noalloc_error().decode()
        assert torch.equal(got, ref)
        assert int((ref >= 0).sum()) > 0


def test_noalloc_at_the_exact_limits():
    """nx + ny + nz and the seed count at their maxima: the coordinate and the
    seed / weight slices then reach the last element of the array."""
    import torch
    from pefdtd import specimen
    L, capi = _lib()
    rng = np.random.default_rng(23)
    nx = 12288 - 2
    xs = np.ascontiguousarray((np.arange(nx) - (nx - 1) / 2) * 1e-6)
    ys = np.zeros(1)
    zs = np.zeros(1)
    R = 4e-3
    seeds = np.ascontiguousarray(specimen.seed_points(R, 2e-3, 16384, rng))
    w = np.ascontiguousarray(rng.uniform(0, 3e-7, len(seeds)))
    for weights in (w, None):
        ref = torch.full((1, 1, nx), -7, dtype=torch.int32, device="cuda")
        got = torch.full_like(ref, -9)
        capi.check(_call(L.pe_label_cylinder, capi, xs, ys, zs, R, seeds, weights, ref))
        for _ in range(2):
            got.fill_(-9)
            rc = _call(L.pe_label_cylinder_noalloc, capi, xs, ys, zs, R, seeds, weights, got)
            assert rc == 0, L.pe_label_cylinder_noalloc_error().decode()
            assert torch.equal(got, ref)
        assert int((ref >= 0).sum()) > 0


def test_noalloc_refuses_oversized_requests():
    import torch
    L, capi = _lib()
    xs = np.zeros(13000)
    seeds = np.zeros((5, 3))
    out = torch.empty(1, dtype=torch.int32, device="cuda")
    rc = _call(L.pe_label_cylinder_noalloc, capi, xs, xs[:1], xs[:1], 1.0, seeds, None, out)
    assert rc == capi.PE_ERR_INVALID
    assert b"exceeds" in L.pe_label_cylinder_noalloc_error()
    many = np.zeros((20000, 3))
    rc = _call(L.pe_label_cylinder_noalloc, capi, xs[:4], xs[:4], xs[:4], 1.0, many, None, out)
    assert rc == capi.PE_ERR_INVALID
