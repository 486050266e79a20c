"""Staggered-grid stencil coefficients and the CFL limit.

Restates sim/core/fdtd.py:45-156 (taylor_coeffs, optimised_coeffs,
ppw_for_error, cfl_limit). The dispersion-optimised tables come out of a
multistart Nelder-Mead solve whose last digits depend on the SciPy build, so
the tables the reference's production runs use are frozen here (values
produced by the reference's own ``optimised_coeffs`` with numpy 2.3.5 / scipy
1.18.1; tests/golden/coeffs.json pins them) and anything else is solved on
demand with the same objective.
"""
from __future__ import annotations

import numpy as np

# (order, kh_max, multistart) -> coefficients, solved by the reference's
# optimised_coeffs (sim/core/fdtd.py:63-132).
_FROZEN = {
    (8, 1.6, True): (1.2170045621116068, -0.09314926512449064, 0.014787497465769746,
                     -0.001642036295283373),
    (8, 2.0, True): (1.2288449375541626, -0.101787967387243, 0.019094796294987997,
                     -0.0027078595524819317),
    (8, 1.6, False): (1.2011233221634154, -0.08171960301730119, 0.009193784243791515,
                      -0.0002762049043527693),
}


def taylor_coeffs(order):
    """Coefficients making sum_k c_k sin((k - 1/2) t) match t/2 to O(t^order)."""
    n = order // 2
    k = np.arange(1, n + 1)
    A = np.array([(2 * k - 1) ** (2 * r + 1) for r in range(n)], float)
    b = np.zeros(n)
    b[0] = 1.0
    return np.linalg.solve(A, b)


def _solve_optimised(order, kh_max, n_grid, multistart):
    from scipy.optimize import minimize
    n = order // 2
    kh = np.linspace(1e-3, kh_max, n_grid)
    K = np.stack([2.0 * np.sin((j + 0.5) * kh) for j in range(n)], axis=1)
    w = 2.0 * (np.arange(n) + 0.5)
    c0 = taylor_coeffs(order)
    if n == 1:
        return c0

    def expand(free):
        c = np.empty(n)
        c[1:] = free
        c[0] = (1.0 - w[1:] @ free) / w[0]
        return c

    def worst(free):
        return np.max(np.abs(K @ expand(free) - kh) / kh)

    if not multistart:
        r = minimize(worst, c0[1:], method="Nelder-Mead",
                     options=dict(maxiter=40000, maxfev=40000, xatol=1e-13, fatol=1e-15))
        return expand(r.x) if worst(r.x) < worst(c0[1:]) else c0
    best, bx = worst(c0[1:]), c0[1:]
    rng = np.random.default_rng(0)
    starts = [c0[1:]] + [c0[1:] * (1.0 + 0.15 * rng.standard_normal(n - 1)) for _ in range(24)]
    for s in starts:
        r = minimize(worst, s, method="Nelder-Mead",
                     options=dict(maxiter=40000, maxfev=40000, xatol=1e-14, fatol=1e-16))
        r = minimize(worst, r.x, method="Nelder-Mead",
                     options=dict(maxiter=40000, maxfev=40000, xatol=1e-14, fatol=1e-16))
        if worst(r.x) < best:
            best, bx = worst(r.x), r.x
    return expand(bx)


def optimised_coeffs(order, kh_max=1.6, n_grid=400, multistart=True):
    """Peak-phase-error-optimised staggered coefficients (long-wave exact)."""
    key = (int(order), float(kh_max), bool(multistart))
    if n_grid == 400 and key in _FROZEN:
        return np.array(_FROZEN[key])
    return _solve_optimised(order, kh_max, n_grid, multistart)


def ppw_for_error(c, tol=1e-3, kh_hi=3.0):
    kh = np.linspace(1e-3, kh_hi, 3000)
    keff = sum(2.0 * c[j] * np.sin((j + 0.5) * kh) for j in range(len(c)))
    ok = kh[np.abs(keff - kh) / kh < tol]
    return float(2 * np.pi / ok.max()) if len(ok) else np.inf


def cfl_limit(c, dim=3):
    """dt <= cfl_limit * h / v_max for the staggered scheme."""
    return 1.0 / (np.sqrt(dim) * np.sum(np.abs(np.asarray(c, float))))
