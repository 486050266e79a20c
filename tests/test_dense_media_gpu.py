"""Per-cell media on the dense entry points (forward_fused / forward).

The reference's dense path takes 21 arbitrary stiffness maps
(sim/core/fdtd.py:236-376, kernels K1-K3 :392-583), e.g. a per-voxel c-axis
field (vendor/ringfwi/axisfield.py:104-120). Media with more distinct cells
than a material table holds run on the per-cell kernel variant (table row =
cell): bit-exact against the oracle with the product's FMA placement in FP32
and FP64, within 1e-5 of the reference's own dense kernels; and a medium that
also fits a table gives the same bits either way.
"""
import numpy as np
import pytest

from helpers import make_small, rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _axis_field_medium(shape, seed=3):
    """A smoothly varying c-axis in every ice voxel of a cylinder (each voxel
    its own medium), couplant outside: the per-voxel form of a fabric."""
    from pefdtd.materials import stiffness_maps
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r2 = (x - (nx - 1) / 2) ** 2 + (y - (ny - 1) / 2) ** 2
    ice = (r2 <= (0.4 * min(nx, ny)) ** 2) & (z >= 3) & (z < nz - 3)
    rng = np.random.default_rng(seed)
    k = rng.uniform(0.1, 0.3, 3)
    theta = 0.6 + 0.4 * np.sin(k[0] * x + k[1] * z)
    phi = 1.0 + 0.8 * np.cos(k[2] * y - k[0] * z)
    lab = np.full(shape, -1, np.int64)
    lab[ice] = np.arange(int(ice.sum()))
    t, p = theta[ice], phi[ice]
    axes = np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], axis=1)
    C, rho = stiffness_maps(lab, axes)
    return C, rho, int(ice.sum())


def _probe(shape):
    nz, ny, nx = shape
    pts = [(3, ny // 2 + dy, nx // 2 + dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    w = 1.0 / len(pts)
    return [(q, w) for q in pts], [(pts, np.full(len(pts), w))]


def _oracle_problem(C, rho, h, dt, nt, src, rec, wav, coeffs, sponge, dtype, record):
    """The same medium as an oracle problem with one table row per cell."""
    from pefdtd import damping
    from pefdtd.fdtd import _flat_probe, _media_rows, _rows_to_tables
    rows, shape = _media_rows(C, rho)
    Ct, rho_t = _rows_to_tables(rows, dtype)
    s_idx, s_w, r_off, r_idx, r_w = _flat_probe(shape, src, rec, dtype)
    cast = np.dtype(dtype).type
    return dict(mats=np.arange(rows.shape[0], dtype=np.int32).reshape(shape), Ct=Ct, rho_t=rho_t,
                damp=damping.sponge_profile(shape, sponge), coeffs=np.asarray(coeffs, dtype),
                inv_h=cast(1.0 / h), dt=cast(dt), dt_h=cast(dt / h), src_idx=s_idx, src_w=s_w,
                rec_off=r_off, rec_idx=r_idx, rec_w=r_w, wavelet=np.asarray(wav, dtype)[:nt], nt=nt,
                record=record, damped_record=True)


@pytest.mark.parametrize("record", ["vz", "pressure"])
def test_per_voxel_axis_field_bit_exact_and_vs_reference_dense(record):
    from pefdtd import fdtd
    from pefdtd.coeffs import optimised_coeffs
    shape = (28, 40, 40)
    C, rho, n_ice = _axis_field_medium(shape)
    assert n_ice > 16383                     # more media than a table holds
    h, nt = 2e-4, 160
    coeffs = optimised_coeffs(8)
    dt = 0.5 * 0.42 * h / 5000.0          # below the face-density speed bound of ice on couplant
    wav = np.sin(2 * np.pi * 1e6 * np.arange(nt) * dt) * np.exp(-((np.arange(nt) - 40) / 15.0) ** 2)
    src, rec = _probe(shape)
    tr = fdtd.forward_fused(C, rho, h, dt, nt, src, wav, rec, coeffs=coeffs, sponge_width=3, record=record)
    pr = _oracle_problem(C, rho, h, dt, nt, src, rec, wav, coeffs, 3, np.float32, record)
    ref = O.run_oracle(pr, fma_mode=1)
    assert np.abs(ref).max() > 0
    assert np.array_equal(tr, ref), f"max |diff| {np.abs(tr - ref).max()}"
    tr64 = fdtd.forward_fused(C, rho, h, dt, nt, src, wav, rec, coeffs=coeffs, sponge_width=3,
                              record=record, dtype="float64")
    pr64 = _oracle_problem(C, rho, h, dt, nt, src, rec, wav, coeffs, 3, np.float64, record)
    assert np.array_equal(tr64, O.run_oracle(pr64, dtype=np.float64, fma_mode=1))
    assert rel_l2(tr, tr64) < TOL
    if O.ref_lib() is not None:
        assert rel_l2(tr, O.run_reference_dense(pr)) < TOL


def test_table_and_per_cell_media_give_the_same_bits():
    from pefdtd import fdtd
    from pefdtd.materials import stiffness_maps
    p = make_small(nt=90, shape=(18, 22, 24), n_grains=6, sponge=3)
    C, rho = stiffness_maps(p["lab"], p["axes"])
    args = (C, rho, p["h"], p["dt"], p["nt"], p["src_pts"], p["wavelet"], p["rec_groups"])
    for dtype in ("float32", "float64"):
        a = fdtd.forward_fused(*args, coeffs=p["coeffs"], sponge_width=3, record="vz", dtype=dtype,
                               media="table")
        b = fdtd.forward_fused(*args, coeffs=p["coeffs"], sponge_width=3, record="vz", dtype=dtype,
                               media="dense")
        assert np.abs(a).max() > 0
        assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        fdtd.forward_fused(*args, media="bogus")
