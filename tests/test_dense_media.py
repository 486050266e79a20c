"""Per-cell media on the CPU (pefdtd.fdtd._compress_dense): the entry points
that take a per-cell stiffness dict (forward_fused, forward) fold it into
table rows when the distinct media fit the label table, else run one row per
cell (the per-cell kernel variant); either way every cell keeps its exact
stiffness and density."""
import numpy as np
import pytest

import helpers  # noqa: F401  (puts the package on sys.path)

KEYS = [(i, j) for i in range(6) for j in range(i, 6)]


def _media(shape, n_distinct, seed):
    """A per-cell C dict and density: n_distinct media (None: every cell its own)."""
    rng = np.random.default_rng(seed)
    ncell = int(np.prod(shape))
    if n_distinct is None:
        rows = rng.uniform(1e9, 2e10, size=(ncell, 22))
    else:
        rows = rng.uniform(1e9, 2e10, size=(n_distinct, 22))[rng.integers(0, n_distinct, size=ncell)]
    rows[:, 21] = rng.uniform(300.0, 1000.0, size=ncell) if n_distinct is None else rows[:, 21] * 1e-7
    C = {f"C{i + 1}{j + 1}": rows[:, k].reshape(shape) for k, (i, j) in enumerate(KEYS)}
    return C, rows[:, 21].reshape(shape), rows


def _per_cell(mats, Ct, rho_t, shape):
    Ct = np.asarray(Ct, float).reshape(-1, 6, 6)
    return Ct[mats.reshape(-1)], np.asarray(rho_t, float)[mats.reshape(-1)]


def test_few_media_fold_into_table_rows():
    from pefdtd.fdtd import _compress_dense
    shape = (6, 7, 8)
    C, rho, rows = _media(shape, 5, seed=1)
    mats, Ct, rho_t, variant = _compress_dense(C, rho, np.float64)
    assert variant is None and mats.dtype == np.uint16 and len(rho_t) == 5
    Cc, rc = _per_cell(mats, Ct, rho_t, shape)
    for k, (i, j) in enumerate(KEYS):
        assert np.array_equal(Cc[:, i, j], rows[:, k]) and np.array_equal(Cc[:, j, i], rows[:, k])
    assert np.array_equal(rc, rows[:, 21])


def test_more_media_than_a_table_holds_run_one_row_per_cell():
    from pefdtd import _capi
    from pefdtd.fdtd import _compress_dense
    shape = (20, 30, 30)                          # 18000 distinct media > the table's rows
    assert np.prod(shape) > _capi.MAX_MATERIALS
    C, rho, rows = _media(shape, None, seed=2)
    mats, Ct, rho_t, variant = _compress_dense(C, rho, np.float32)
    assert variant == "dense" and not mats.any() and len(rho_t) == np.prod(shape)
    Ct = np.asarray(Ct).reshape(-1, 6, 6)
    for k, (i, j) in enumerate(KEYS):           # row n is cell n (C order), rounded to the working type
        assert np.array_equal(Ct[:, i, j], rows[:, k].astype(np.float32))
    assert np.array_equal(rho_t, rows[:, 21].astype(np.float32))
    with pytest.raises(ValueError, match="exceed"):
        _compress_dense(C, rho, np.float32, media="table")
    m2, _, _, v2 = _compress_dense(*_media((4, 4, 4), 3, seed=3)[:2], np.float32, media="dense")
    assert v2 == "dense" and m2.shape == (4, 4, 4)
    with pytest.raises(ValueError, match="media must be"):
        _compress_dense(C, rho, np.float32, media="cells")
