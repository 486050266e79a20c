"""The preconditions of the pair kernels' unguarded bodies (CPU).

k_stress_pair and k_velocity_pair (pe_kernels_pair.cuh) run tiles that pass
pair_tile_inside / pair_vtile_inside with every x / y tap limit and
neighbour guard compiled out, and the stress kernel's z-interior planes
(T_H <= q <= nz - 1 - T_H) with the z limits and move guards compiled out as
well. That is exact only if, in such a tile or plane, every tap of the
order-8 stencil (four per side) and every neighbour a move or a face
density reads exists. This checks it for every tile of every even grid width
up to 400 (the pair kernels need 16-byte rows), restating the guards from
the kernels, with the tile constants read from the headers."""
import os
import re

import helpers  # noqa: F401  (puts the package on sys.path)

CSRC = os.path.join(helpers.PKG, "pefdtd", "csrc")


def const(name, src):
    m = re.search(r"\b" + name + r"\s*=\s*([^,;]+)[,;]", src)
    assert m, name
    return m.group(1).strip()


def constants():
    pair = open(os.path.join(CSRC, "pe_kernels_pair.cuh")).read()
    tiled = open(os.path.join(CSRC, "pe_kernels_tiled.cuh")).read()
    c = dict(T_H=int(const("T_H", tiled)), PR_LX=int(const("PR_LX", pair)),
             PS_ROWS=int(const("PS_ROWS", pair)), PS_OX=int(const("PS_OX", pair)),
             PS_GW=int(const("PS_GW", pair)), PV_ROWS=int(const("PV_ROWS", pair)),
             PV_OX=int(const("PV_OX", pair)))
    assert const("PS_OY", pair) == "PS_ROWS - 2" and const("PV_OY", pair) == "PV_ROWS"
    c["PS_OY"], c["PV_OY"] = c["PS_ROWS"] - 2, c["PV_ROWS"]
    return c


def lim_b(i, n):
    return min(i, n - i)


def lim_f(i, n):
    return min(i + 1, n - i - 1)


def all_taps(i, n, T_H):
    """Every tap j < T_H of both difference directions exists at i."""
    return lim_b(i, n) >= T_H and lim_f(i, n) >= T_H


def test_stress_tiles_inside_need_no_x_y_guards():
    c = constants()
    T_H, OX, OY, GW, ROWS = c["T_H"], c["PS_OX"], c["PS_OY"], c["PS_GW"], c["PS_ROWS"]
    for n in range(8, 401, 2):
        for b in range(n // OX + 3):
            S0 = b * OX - 2                       # first strain column (row: b * OY - 1)
            if S0 - T_H >= 0 and S0 + GW - 1 + T_H < n:          # pair_tile_inside, x part
                for x in range(S0, S0 + GW):
                    assert all_taps(x, n, T_H) and 1 <= x <= n - 2, (n, b, x)
            S0y = b * OY - 1
            if S0y - T_H >= 0 and S0y + ROWS - 1 + T_H < n:      # pair_tile_inside, y part
                for y in range(S0y, S0y + ROWS):
                    assert all_taps(y, n, T_H) and 1 <= y <= n - 2, (n, b, y)


def test_velocity_tiles_inside_need_no_x_y_guards():
    c = constants()
    T_H, OX, OY = c["T_H"], c["PV_OX"], c["PV_OY"]
    for n in range(8, 401, 2):
        for b in range(n // min(OX, OY) + 2):
            x0 = b * OX
            if x0 - T_H >= 0 and x0 + OX - 1 + T_H < n:          # pair_vtile_inside, x part
                for x in range(x0, x0 + OX):
                    assert all_taps(x, n, T_H), (n, b, x)
                    assert x + 1 < n                              # the +x face-density neighbour
                assert x0 + OX - 1 < n - 1                         # cell 1 of the last pair: xin1
            y0 = b * OY
            if y0 - T_H >= 0 and y0 + OY - 1 + T_H < n:          # pair_vtile_inside, y part
                for y in range(y0, y0 + OY):
                    assert all_taps(y, n, T_H) and y < n - 1, (n, b, y)   # yin


def test_stress_z_interior_planes_need_no_z_guards():
    """Strain plane q with T_H <= q <= nz - 1 - T_H: all z taps exist, and
    the plane it updates, z = q - 1, has both z neighbours for its moves."""
    T_H = constants()["T_H"]
    for nz in range(2, 400):
        for q in range(T_H, nz - T_H):
            assert all_taps(q, nz, T_H), (nz, q)
            z = q - 1
            assert 1 <= z <= nz - 2, (nz, q)
