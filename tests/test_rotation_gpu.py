"""The azimuth rotation on the device (pe_rotated_grid) reproduces the host
restatement of the reference's rotated_grid (sim/core/rotation_test.py:60-137)
bit for bit: integer labels and indexing are exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("h_ratio", [1.0, 0.8, 1.37])
def test_rotated_grid_device_bit_exact(h_ratio):
    from pefdtd import specimen
    rng = np.random.default_rng(7)
    nx_s, nz_s, h_spec = 61, 23, 0.25e-3
    lab = rng.integers(-1, 40, size=(nx_s, nx_s, nz_s)).astype(np.int32)
    axes = rng.normal(size=(40, 3))
    h = h_spec * h_ratio
    for rot in (0.0, 10.0, 45.0, 90.0, 137.5, 180.0, 271.3, 350.0):
        a, nd, m, ax = specimen.rotated_grid(lab, axes, h_spec, h, 5, rot)
        b, nd2, m2, ax2 = specimen.rotated_grid_device(lab, axes, h_spec, h, 5, rot)
        assert (nd, m) == (nd2, m2)
        assert np.array_equal(a, b.cpu().numpy()), rot
        assert np.array_equal(ax, ax2)
