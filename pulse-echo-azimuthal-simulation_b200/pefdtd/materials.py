"""Per-material stiffness and density tables for the label-indexed solver.

Material 0 is the fluid couplant (specimen label -1) and material m is grain
m-1, as in the reference's ``material_tables``
(sim/core/fdtd.py:1580-1603, which calls
vendor/ringfwi/anisotropy.py:418-456). Each grain carries the transversely
isotropic single-crystal ice tensor (vendor/ringfwi/anisotropy.py:356-370,
C11 13.93, C33 15.01, C44 3.01, C12 7.08, C13 5.77 GPa, rho 917) rotated so
its symmetry axis lies along the grain's c-axis.

The rotation here is the 6x6 Bond transformation C' = M C M^T of the
Rodrigues rotation that takes z onto the c-axis
(vendor/ringfwi/anisotropy.py:339-353). The reference rotates the
fourth-order tensor with an einsum (:332-336); both are the same linear map,
so the f32 tables agree to the last bit except at rare rounding ties
(checked against the reference's own tables in tests/test_host_setup.py).
"""
from __future__ import annotations

import numpy as np

ICE = dict(C11=13.93e9, C33=15.01e9, C44=3.01e9, C12=7.08e9, C13=5.77e9, rho=917.0)

# Voigt index -> tensor index pair (engineering shear strain convention)
_VOIGT = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))

# upper-triangle (I <= J) order of the 21 independent constants, row major
C21_INDEX = [(i, j) for i in range(6) for j in range(i, 6)]
C21_KEYS = [f"C{i + 1}{j + 1}" for i, j in C21_INDEX]


def ti_stiffness_6(C11, C33, C44, C12, C13, **_):
    """6x6 Voigt stiffness of a TI solid with its symmetry axis along z."""
    C66 = 0.5 * (C11 - C12)
    C = np.zeros((6, 6))
    C[0, 0] = C[1, 1] = C11
    C[2, 2] = C33
    C[0, 1] = C[1, 0] = C12
    C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = C13
    C[3, 3] = C[4, 4] = C44
    C[5, 5] = C66
    return C


def rotation_z_to(axis):
    """Rotation matrix taking +z onto the unit vector ``axis`` (Rodrigues).

    Antiparallel axes map to diag(1, -1, -1), as in
    vendor/ringfwi/anisotropy.py:339-353.
    """
    a = np.asarray(axis, float)
    a = a / np.linalg.norm(a)
    v = np.array([-a[1], a[0], 0.0])            # z x a
    c = float(a[2])                             # z . a
    if np.linalg.norm(v) < 1e-12:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    K = np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])
    return np.eye(3) + K + K @ K / (1.0 + c)


def bond_matrix(R):
    """6x6 stress-transformation (Bond) matrix of rotation R: C' = M C M^T.

    Row a, column b of M is the coefficient of stress component b in rotated
    stress component a, with tensor pairs taken from the Voigt map above.
    """
    R = np.asarray(R, float)
    M = np.empty(R.shape[:-2] + (6, 6))
    for a, (i, j) in enumerate(_VOIGT):
        for b, (k, l) in enumerate(_VOIGT):
            if k == l:
                M[..., a, b] = R[..., i, k] * R[..., j, l]
            else:
                M[..., a, b] = R[..., i, k] * R[..., j, l] + R[..., i, l] * R[..., j, k]
    return M


def rotate_voigt(C6, R):
    """Rotate a 6x6 Voigt stiffness by rotation matrix (or stack) R."""
    M = bond_matrix(R)
    return M @ np.asarray(C6, float) @ np.swapaxes(M, -1, -2)


def grain_stiffness(axes, material=None):
    """(n, 6, 6) rotated stiffness for each c-axis in ``axes`` (n, 3)."""
    mat = ICE if material is None else material
    C0 = ti_stiffness_6(**mat)
    axes = np.atleast_2d(np.asarray(axes, float))
    R = np.stack([rotation_z_to(a) for a in axes]) if len(axes) else np.zeros((0, 3, 3))
    return rotate_voigt(C0, R)


def material_tables(axes, c_couplant=1500.0, rho_couplant=300.0, material=None):
    """(Ct (n_mat, 36) f32, rho_t (n_mat,) f32) with row 0 the fluid couplant.

    Same contract as the reference's ``material_tables``
    (sim/core/fdtd.py:1580-1603): the fluid carries only its bulk modulus
    K = rho c^2 in the normal block, zero shear.
    """
    mat = ICE if material is None else material
    axes = np.asarray(axes, float).reshape(-1, 3)
    n_mat = len(axes) + 1
    C = np.zeros((n_mat, 6, 6))
    K = rho_couplant * c_couplant * c_couplant
    C[0, :3, :3] = K
    if len(axes):
        C[1:] = grain_stiffness(axes, mat)
    # symmetric by construction; enforce exact symmetry of the f32 rows
    iu = np.triu_indices(6)
    Cs = C.copy()
    Cs[:, iu[1], iu[0]] = C[:, iu[0], iu[1]]
    Ct = Cs.reshape(n_mat, 36).astype(np.float32)
    rho_t = np.full(n_mat, float(mat["rho"]))
    rho_t[0] = rho_couplant
    return Ct, rho_t.astype(np.float32)


def stiffness_maps(labels, axes, c_couplant=1500.0, rho_couplant=300.0, material=None):
    """Per-cell dict of the 21 Voigt maps ("C11".."C66") and density for a
    label volume (-1 = couplant), the input form of the dense entry points
    (what vendor/ringfwi/anisotropy.py:418-456 builds)."""
    labels = np.asarray(labels)
    mat = ICE if material is None else material
    axes = np.asarray(axes, float).reshape(-1, 3)
    n_mat = len(axes) + 1
    C = np.zeros((n_mat, 6, 6))
    C[0, :3, :3] = rho_couplant * c_couplant * c_couplant
    if len(axes):
        C[1:] = grain_stiffness(axes, mat)
    m = labels + 1
    maps = {k: C[:, i, j][m] for k, (i, j) in zip(C21_KEYS, C21_INDEX)}
    rho_t = np.full(n_mat, float(mat["rho"]))
    rho_t[0] = rho_couplant
    return maps, rho_t[m]


def c36_to_c21(Ct):
    """(n_mat, 36) symmetric rows -> (n_mat, 21) upper triangle, row major."""
    Ct = np.asarray(Ct).reshape(-1, 6, 6)
    return np.stack([Ct[:, i, j] for i, j in C21_INDEX], axis=1)


def c21_to_c36(C21):
    C21 = np.asarray(C21)
    out = np.zeros((C21.shape[0], 6, 6), C21.dtype)
    for k, (i, j) in enumerate(C21_INDEX):
        out[:, i, j] = C21[:, k]
        out[:, j, i] = C21[:, k]
    return out.reshape(-1, 36)
