"""Grid crops (pefdtd.crop): the reference's causal-crop and E1-corridor
index arithmetic (sim/fw_checks/fw_crop_validate.py:71-75,
fw_e1_corridor_validate.py:79-83), probe shifts and cost ratios, on CPU."""
import numpy as np

from helpers import synthetic_echo  # noqa: F401  (puts the package on sys.path)
from pefdtd import crop


def _grid():
    rng = np.random.default_rng(2)
    lab = rng.integers(-1, 5, size=(30, 80, 120)).astype(np.int32)
    dm = rng.uniform(0.5, 1, size=lab.shape).astype(np.float32)
    return lab, dm


def test_causal_crop_matches_reference_cut_on_the_rim_probe_axis():
    lab, dm = _grid()
    h, dt, t_keep = 0.2e-3, 3e-8, 8e-6
    ixp = 110
    pts = [(15 + a, 40 + b, ixp) for a in (-1, 0, 1) for b in (-2, 0, 2)]
    out = crop.causal_crop(lab, pts, h, dt, t_keep, damp_mask=dm)
    R = crop.C_CAUSAL * t_keep / 2 + crop.MARGIN
    ix0 = max(int(ixp - R / h) - 1, 0)            # the reference's cut
    assert out["offset"][2] == ix0
    z0, y0, x0 = out["offset"]
    assert np.array_equal(out["lab"], lab[z0:z0 + out["lab"].shape[0], y0:y0 + out["lab"].shape[1], x0:])
    assert np.array_equal(out["damp_mask"], dm[z0:z0 + out["lab"].shape[0], y0:y0 + out["lab"].shape[1], x0:])
    for (a, b, c), (a2, b2, c2) in zip(pts, out["pts"]):
        assert (a - z0, b - y0, c - x0) == (a2, b2, c2)
        assert lab[a, b, c] == out["lab"][a2, b2, c2]
    assert out["nt"] == int(t_keep / dt)
    assert crop.cost_ratio(lab.shape, out["lab"].shape, 400, out["nt"]) < 1


def test_e1_corridor_matches_reference_rows():
    lab, dm = _grid()
    h, hw = 0.2e-3, 3e-3
    cy = lab.shape[1] // 2
    pts = [(15, cy + b, 100) for b in (-3, 0, 3)]
    out = crop.e1_corridor(lab, pts, h, hw, damp_mask=dm)
    ky = int(hw / h)
    assert out["offset"] == (0, cy - ky, 0)
    assert np.array_equal(out["lab"], lab[:, cy - ky:cy + ky + 1, :])
    assert np.array_equal(out["damp_mask"], dm[:, cy - ky:cy + ky + 1, :])
    assert [p[1] for p in out["pts"]] == [ky - 3, ky, ky + 3]
