"""Coefficients of the phase polynomials of the regular kernels.

FP32 (mixed-precision kernels, tiles.cuh):
cos t ~ 1 + c1 z + c2 z^2 + ... and sin t ~ t (1 + s1 z + s2 z^2 + ...), z = t^2, on
|t| <= T, fitted by discrete minimax (a linear program over 6001 points of [0, T]; both
functions have the symmetry of the form, so [0, T] suffices).

    python fit_phase_polys.py [tmax ncos nsin]

Default: |t| <= 0.8 with cos of degree 8 and sin of degree 7 (ncos = 4, nsin = 3 terms
beyond the leading one; max errors 6.5e-11 and 2.1e-9, below FP32 rounding), the
coefficients of poly_cos_sin / poly_cos_sin2, used by launches with
k (max rad_x + max rad_y) <= 0.8 and, after a reduction by pi/2, by every other phase.

FP64 (sincos_small in common.cuh, the pair-referenced phases of the FP64 kernels):

    python fit_phase_polys.py fp64

cos t ~ 1 + z P(z) and sin t ~ t + t z Q(z), z = t^2, P and Q of degree 5 on |t| <= 0.8,
by Chebyshev interpolation of (cos(sqrt z) - 1) / z and (sin(sqrt z) / sqrt z - 1) / z on
[0, 0.64] at 50 digits (mpmath.chebyfit, near-minimax); the script prints the
coefficients rounded to double and the max errors of cos and sin with them.
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


def fit_fp64(tmax=0.8, degree=5):
    """cos t ~ 1 + z P(z) and sin t ~ t + t z Q(z), z = t^2, on |t| <= tmax, P and Q of
    degree `degree`: their coefficients rounded to double (highest degree first) and the
    max abs errors of cos and sin with the rounded coefficients."""
    import mpmath as mp

    mp.mp.dps = 50
    zmax = mp.mpf(tmax) ** 2

    def pc(z):
        return (mp.cos(mp.sqrt(z)) - 1) / z if z != 0 else mp.mpf(-0.5)

    def ps(z):
        return (mp.sin(mp.sqrt(z)) / mp.sqrt(z) - 1) / z if z != 0 else -mp.mpf(1) / 6

    out = {}
    for name, f, g in (("cos", pc, lambda z, v: 1 + z * v - mp.cos(mp.sqrt(z))),
                       ("sin", ps, lambda z, v: mp.sqrt(z) * (1 + z * v) - mp.sin(mp.sqrt(z)))):
        coef = [float(c) for c in mp.chebyfit(f, [0, zmax], degree + 1)]
        err = 0
        for i in range(4001):
            z = zmax * i / 4000
            err = max(err, abs(g(z, mp.polyval([mp.mpf(c) for c in coef], z))))
        out[name] = (coef, float(err))
    return out


if __name__ == "__main__":
    import sys

    if len(sys.argv) == 2 and sys.argv[1] == "fp64":
        for name, (coef, err) in fit_fp64().items():
            print(f"{name}: max abs error {err:.2e}; coefficients z^5 .. z^0:")
            print("  " + ", ".join(f"{c!r}" for c in coef))
        sys.exit(0)
    args = [float(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3])] if len(sys.argv) == 4 else [0.8, 4, 3]
    for tmax, nc, ns in (tuple(args),):
        c, ec, s, es = fit(tmax, nc, ns)
        print(f"|t| <= {tmax}: cos degree {2 * nc}, max error {ec:.2e}; "
              f"sin degree {2 * ns + 1}, max error {es:.2e}")
        print("  cos z^1..: " + ", ".join(f"{v:.9e}" for v in c))
        print("  sin z^1..: " + ", ".join(f"{v:.9e}" for v in s))
