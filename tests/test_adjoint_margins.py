"""The margins behind the adjoint's unguarded instantiations (CPU).

The adjoint kernels (pe_adjoint.cuh) compile every guard out in blocks whose
cells lie ADJ_MARGIN_LO or more cells inside the low faces and ADJ_MARGIN_HI
or more inside the high ones, per axis. That is exact only if every guard
holds there. The guards are restated here from the kernels (each a
transcription of the forward tap and move conditions) and checked for every
position inside the margins on every axis length that has one, at the
largest stencil (taps j = 0..3). The two constants are read from the header,
so a change there is checked too."""
import os
import re

import helpers  # noqa: F401  (puts the package on sys.path)

HDR = os.path.join(helpers.PKG, "pefdtd", "csrc", "pe_adjoint.cuh")


def margins():
    src = open(HDR).read()
    m = re.search(r"constexpr int ADJ_MARGIN_LO = (\d+), ADJ_MARGIN_HI = (\d+);", src)
    assert m, "margin constants not found in pe_adjoint.cuh"
    return int(m.group(1)), int(m.group(2))


def gF(x, j, n):      # forward-difference tap j exists at x
    return j <= x < n - j - 1


def gB(x, j, n):      # backward-difference tap j exists at x
    return j + 1 <= x < n - j


def move_axis_ok(x, d, n):
    """One axis of move_ok: the forward cell x exists and, for a move with a
    component d along the axis, has its neighbour on that side."""
    if not 0 <= x < n:
        return False
    if d > 0 and x > n - 2:
        return False
    if d < 0 and x < 1:
        return False
    return True


def guards_at(y, n):
    """Every guard the adjoint kernels evaluate for a cell at y on an axis of
    length n, for taps j = 0..3 and move offsets a, d in {-1, 0, 1}."""
    out = []
    for j in range(4):
        out += [gF(y - j - 1, j, n), gF(y + j, j, n)]          # DfT: forward cells y - j - 1, y + j
        out += [gB(y - j, j, n), gB(y + j + 1, j, n)]          # DbT: forward cells y - j, y + j + 1
        out += [gB(y, j, n), gF(y, j, n)]                      # forward strains at the cell
    for d in (-1, 0, 1):
        out.append(move_axis_ok(y, d, n))                      # moves at the cell (adj_q)
        for a in (-1, 0, 1):
            out.append(move_axis_ok(y - a, d, n))              # transposed moves (adj_t)
    return out


def test_every_guard_holds_inside_the_margins():
    lo, hi = margins()
    for n in range(lo + hi, 200):
        for y in range(lo, n - hi + 1):
            assert all(guards_at(y, n)), (n, y)


def test_the_margins_are_tight_for_the_derivative_transposes():
    """One cell closer to either face, some guard fails: the margins are the
    smallest that compile every guard out at order 8."""
    lo, hi = margins()
    for n in range(lo + hi + 2, 120):
        assert not all(guards_at(lo - 1, n))
        assert not all(guards_at(n - hi + 1, n))
