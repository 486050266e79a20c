"""Cheaper solves by cropping the grid: the causal coda crop and the E1 beam
corridor.

Both are transformations of the problem before the solve (labels, damping
mask and probe cells cut to a sub-box, probe shifted), run with the same
solver; the reference applies them in sim/fw_checks/fw_crop_validate.py
(causal crop, ~0.45x cost at 5 MHz) and sim/fw_checks/fw_e1_corridor_validate.py
(E1 corridor, ~0.55x cells), licensed by measurement against uncropped runs.

* Causal crop: for a monostatic probe, cells farther than
  R = c_causal * t_keep / 2 + margin from the probe cannot influence the
  trace before t_keep, so they are dropped (c_causal = 4200 m/s exceeds the
  fastest physical qP speed and the order-8 grid's numerical precursors) and
  the record stops at t_keep. The reference crops the side of the disk away
  from its +x rim probe (`ix0 = max(int(ixp - R/h) - 1, 0)`,
  fw_crop_validate.py:71-75); here every axis is cropped that way on both
  sides of the probe's bounding box, which reduces to the reference's cut for
  its geometry.
* E1 corridor: keeps |y - y_probe| <= half_width about the beam axis
  (`ky = int(half_width/h)`, rows cy - ky .. cy + ky,
  fw_e1_corridor_validate.py:79-83). Not provable by causality; the
  reference accepts it when the E1 amplitude stays within 1 % and its time of
  flight within 20 ns of the full run (:112-116).
"""
from __future__ import annotations

import numpy as np

C_CAUSAL = 4200.0   # m/s, above qP max and the numerical precursor speed
MARGIN = 2e-3       # m


def _cut(arrays, sl):
    return [None if a is None else np.ascontiguousarray(np.asarray(a)[sl]) for a in arrays]


def causal_box(shape, pts, h, t_keep, c_causal=C_CAUSAL, margin=MARGIN):
    """(lo, hi) per axis (z, y, x) of the cells within the causal radius of
    the probe cells `pts` ((iz, iy, ix) tuples)."""
    P = np.asarray(pts, int).reshape(-1, 3)
    R = c_causal * t_keep / 2 + margin
    k = R / h
    lo = [max(int(P[:, a].min() - k) - 1, 0) for a in range(3)]
    hi = [min(int(P[:, a].max() + k) + 2, shape[a]) for a in range(3)]
    return lo, hi


def causal_crop(lab, pts, h, dt, t_keep, damp_mask=None, c_causal=C_CAUSAL, margin=MARGIN):
    """Crop (lab, damp_mask) to the causal box of the probe `pts` for a
    record of t_keep seconds. Returns dict(lab, damp_mask, pts, offset, nt):
    the cropped arrays, the probe cells in cropped coordinates, the (z, y, x)
    offset of the crop and the step count int(t_keep / dt)."""
    lab = np.asarray(lab)
    lo, hi = causal_box(lab.shape, pts, h, t_keep, c_causal, margin)
    sl = tuple(slice(a, b) for a, b in zip(lo, hi))
    lab_c, dm_c = _cut([lab, damp_mask], sl)
    pts_c = [(int(a) - lo[0], int(b) - lo[1], int(c) - lo[2]) for a, b, c in pts]
    return dict(lab=lab_c, damp_mask=dm_c, pts=pts_c, offset=tuple(lo), nt=int(t_keep / dt))


def e1_corridor(lab, pts, h, half_width, damp_mask=None, centre_y=None):
    """Crop (lab, damp_mask) to |y - centre_y| <= half_width (rows
    centre_y - ky .. centre_y + ky, ky = int(half_width / h)); centre_y
    defaults to the grid's middle row, the beam axis of the reference's rim
    probe. Returns dict(lab, damp_mask, pts, offset)."""
    lab = np.asarray(lab)
    ny = lab.shape[1]
    cy = ny // 2 if centre_y is None else int(centre_y)
    ky = int(half_width / h)
    y0, y1 = max(cy - ky, 0), min(cy + ky + 1, ny)
    sl = (slice(None), slice(y0, y1), slice(None))
    lab_c, dm_c = _cut([lab, damp_mask], sl)
    pts_c = [(int(a), int(b) - y0, int(c)) for a, b, c in pts]
    if any(not 0 <= b < y1 - y0 for _, b, _ in pts_c):
        raise ValueError("probe cells fall outside the corridor")
    return dict(lab=lab_c, damp_mask=dm_c, pts=pts_c, offset=(0, y0, 0))


def cost_ratio(full_shape, cropped_shape, nt_full, nt_cropped):
    """Cell updates of the cropped solve over the full one."""
    return (float(np.prod(cropped_shape)) * nt_cropped) / (float(np.prod(full_shape)) * nt_full)
