"""Coefficients of the FP32 phase polynomials of the mixed-precision kernels (tiles.cuh):
cos t ~ 1 + c1 z + c2 z^2 + ... and sin t ~ t (1 + s1 z + s2 z^2 + ...), z = t^2, on
|t| <= T, fitted by discrete minimax (a linear program over 6001 points of [0, T]; both
functions have the symmetry of the form, so [0, T] suffices).

    python fit_phase_polys.py [tmax ncos nsin]

Default: |t| <= 0.8 with cos of degree 8 and sin of degree 7 (ncos = 4, nsin = 3 terms
beyond the leading one; max errors 6.5e-11 and 2.1e-9, below FP32 rounding), the
coefficients of poly_cos_sin / poly_cos_sin2, used by launches with
k (max rad_x + max rad_y) <= 0.8 and, after a reduction by pi/2, by every other phase.
"""

import numpy as np
from scipy.optimize import linprog


def minimax(f, basis, t):
    """min_c max_j |f(t_j) - sum_i c_i basis_i(t_j)|: variables (c, e), minimise e."""
    b = np.stack([g(t) for g in basis], axis=1)
    n = b.shape[1]
    cost = np.zeros(n + 1)
    cost[-1] = 1.0
    ones = np.ones((len(t), 1))
    a_ub = np.vstack([np.hstack([b, -ones]), np.hstack([-b, -ones])])
    b_ub = np.concatenate([f(t), -f(t)])
    res = linprog(cost, A_ub=a_ub, b_ub=b_ub, bounds=[(None, None)] * (n + 1), method="highs")
    assert res.success, res.message
    return res.x[:n], res.x[-1]


def fit_series(f, taylor, powers, tmax, npts=6001):
    """f(t) ~ sum_i a_i t^powers[i]: the Taylor coefficients plus a minimax correction of
    the remainder, fitted in the scaled basis (t / tmax)^p against the remainder scaled to
    unit size (so that the linear program's tolerances do not swamp errors of 1e-10)."""
    t = np.linspace(0.0, tmax, npts)
    rem = f(t) - sum(a * t ** p for a, p in zip(taylor, powers))
    scale = np.abs(rem).max()
    d, e = minimax(lambda x: (f(x) - sum(a * x ** p for a, p in zip(taylor, powers))) / scale,
                   [lambda x, p=p: (x / tmax) ** p for p in powers], t)
    coef = np.array([a + scale * di / tmax ** p for a, di, p in zip(taylor, d, powers)])
    err = np.abs(f(t) - sum(a * t ** p for a, p in zip(coef, powers))).max()
    return coef, err


def fit(tmax, ncos, nsin):
    from math import factorial

    # cos t - 1 = sum_{i=1..ncos} c_i t^(2i);  sin t - t = sum_{i=1..nsin} s_i t^(2i+1)
    cp = [2 * i for i in range(1, ncos + 1)]
    sp = [2 * i + 1 for i in range(1, nsin + 1)]
    c, ec = fit_series(lambda x: np.cos(x) - 1.0, [(-1) ** (p // 2) / factorial(p) for p in cp], cp, tmax)
    s, es = fit_series(lambda x: np.sin(x) - x, [(-1) ** (p // 2) / factorial(p) for p in sp], sp, tmax)
    return c, ec, s, es


if __name__ == "__main__":
    import sys

    args = [float(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3])] if len(sys.argv) == 4 else [0.8, 4, 3]
    for tmax, nc, ns in (tuple(args),):
        c, ec, s, es = fit(tmax, nc, ns)
        print(f"|t| <= {tmax}: cos degree {2 * nc}, max error {ec:.2e}; "
              f"sin degree {2 * ns + 1}, max error {es:.2e}")
        print("  cos z^1..: " + ", ".join(f"{v:.9e}" for v in c))
        print("  sin z^1..: " + ", ".join(f"{v:.9e}" for v in s))
