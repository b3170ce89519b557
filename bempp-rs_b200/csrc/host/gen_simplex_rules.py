"""Generate fully symmetric quadrature rules on the reference triangle.

The regular (non-singular) quadrature of the boundary assembler uses a symmetric
triangle rule selected by its number of points (bempp-rs calls
``ndelement::quadrature::simplex_rule(Triangle, npoints)`` at
src/boundary_assemblers.rs:419,434; the crate's tables are the Witherden--Vincent
rules, README.md:38-46).  Those tables live in an unvendored crate, so this script
derives rules with the same point counts and the same polynomial degree as the
Witherden--Vincent family by solving the moment equations

    sum_i w_i p(x_i, y_i) = integral of p over T    for every polynomial p of degree <= d

on the reference triangle T = (0,0), (1,0), (0,1) (weights sum to its area 1/2), written
in an orthogonal (Dubiner) basis so the Levenberg--Marquardt iteration is well
conditioned.  Orbits: S3 = centroid, S21(a) = barycentric (a, a, 1-2a) and its
permutations, S111(a, b) = (a, b, 1-a-b) and its permutations.  The starting orbit
parameters below were found by a seeded random search with the same solver; this script
only polishes them and checks every rule: points strictly inside T, positive weights, and
monomial moments exact to 1e-15.

For 6 points the degree-4 fully symmetric rule is unique, so it is the Witherden--Vincent
6-point rule up to rounding and point order; larger rules have the Witherden--Vincent
degree but need not be the same point sets.

Run:  python gen_simplex_rules.py > simplex_rules_table.inc
"""

from __future__ import annotations

import math
import sys

import numpy as np

# npoints, degree, (n_S3, n_S21, n_S111), starting orbit parameters
#   S3: w; S21: a, w; S111: a, b, w
RULES = [
    (1, 1, (1, 0, 0), [0.5]),
    (3, 2, (0, 1, 0), [0.16666666666666669, 0.16666666666666657]),
    (6, 4, (0, 2, 0), [0.4459484909159649, 0.11169079483900586, 0.09157621350977069,
                       0.05497587182766095]),
    (7, 5, (1, 2, 0), [0.11249999999999999, 0.4701420641051151, 0.06619707639425311,
                       0.10128650732345633, 0.0629695902724136]),
    (12, 6, (0, 2, 1), [0.2492867451709104, 0.058393137863189684, 0.06308901449150223,
                        0.02542245318510341, 0.3103524510337844, 0.6365024991213987,
                        0.041425537809186785]),
    (15, 7, (0, 3, 1), [0.06444245801079386, 0.026084867311915852, 0.44459255761708477,
                        0.010711544656436965, 0.23994364473663288, 0.061767565601999995,
                        0.6468242963556892, 0.04399513604540739, 0.03405134454815693]),
    (16, 8, (1, 3, 1), [0.07215780383889357, 0.17056930775176024, 0.05160868526735912,
                        0.4592925882927232, 0.047545817133642324, 0.05054722831703099,
                        0.016229248811599036, 0.26311282963463806, 0.7284923929554042,
                        0.013615157087217505]),
    (19, 9, (1, 4, 1), [0.04856789814139939, 0.43708959149293664, 0.038913770502387146,
                        0.04472951339445271, 0.012788837829349017, 0.4896825191987376,
                        0.015667350113569536, 0.18820353561903275, 0.039823869463605124,
                        0.22196298916076568, 0.741198598784498, 0.021641769688644688]),
    (25, 10, (1, 2, 3), [0.04160986849322506, 0.16291311787409474, 0.026325974734122293,
                         0.028503500288387832, 0.005475644170134205, 0.516492619327838,
                         0.33669587527823164, 0.028138639855405597, 0.3633626169945705,
                         0.60732977850085, 0.017697473895769193, 0.033685698680610304,
                         0.8130112461498283, 0.014661432047826117]),
    (33, 12, (0, 5, 3), [0.12757614554158592, 0.01739805646535446, 0.021317350453210412,
                         0.00308313052577951, 0.48821738977380486, 0.012865533220227664,
                         0.2712103850121159, 0.031429112108942545, 0.43972439229446025,
                         0.021846272269019203, 0.6089432357797878, 0.2757132696855142,
                         0.020185778883190467, 0.11625191590759718, 0.8580140335440726,
                         0.008658115554329444, 0.022838332222257028, 0.6958360867878034,
                         0.011178386601151724]),
    (37, 13, (1, 4, 4), [0.033980018293415806, 0.02150968110884315, 0.003026168551769585,
                         0.48907694645253935, 0.01199720096444736, 0.4269414142598004,
                         0.027800983765226675, 0.22137228629183292, 0.029139242559599987,
                         0.024370186901093847, 0.8647077702954428, 0.0074827005525828355,
                         0.3084417608921177, 0.6235459955536756, 0.01732063807042419,
                         0.0051263891023823486, 0.7223577931241879, 0.00479534050177163,
                         0.16359740106785042, 0.08789548303219734, 0.012089519905796903]),
]


def expand(params, n3, n21, n111):
    """Orbit parameters -> barycentric points (npts x 3) and weights."""
    lam, w = [], []
    k = 0
    for _ in range(n3):
        lam.append((1 / 3, 1 / 3, 1 / 3))
        w.append(params[k])
        k += 1
    for _ in range(n21):
        a, wt = params[k], params[k + 1]
        k += 2
        for slot in range(3):
            p = [a, a, a]
            p[slot] = 1 - 2 * a
            lam.append(tuple(p))
            w.append(wt)
    for _ in range(n111):
        a, b, wt = params[k], params[k + 1], params[k + 2]
        k += 3
        v = (a, b, 1 - a - b)
        for perm in [(0, 1, 2), (1, 0, 2), (0, 2, 1), (2, 0, 1), (1, 2, 0), (2, 1, 0)]:
            lam.append(tuple(v[perm[s]] for s in range(3)))
            w.append(wt)
    return np.array(lam), np.array(w)


def jacobi(n, alpha, t):
    """Jacobi polynomials P_0..P_n^{(alpha, 0)}(t) by the three-term recurrence."""
    out = [np.ones_like(t)]
    if n == 0:
        return out
    out.append(0.5 * (alpha + 2) * t + 0.5 * alpha)
    for k in range(1, n):
        a1 = 2 * (k + 1) * (k + alpha + 1) * (2 * k + alpha)
        a2 = (2 * k + alpha + 1) * (alpha * alpha)
        a3 = (2 * k + alpha) * (2 * k + alpha + 1) * (2 * k + alpha + 2)
        a4 = 2 * (k + alpha) * k * (2 * k + alpha + 2)
        out.append(((a2 + a3 * t) * out[-1] - a4 * out[-2]) / a1)
    return out


def dubiner(x, y, deg):
    """Orthogonal polynomial basis on T (collapsed-coordinate construction)."""
    a = 2 * x + y - 1
    b = 1 - y
    q = [np.ones_like(x), a]
    for m in range(1, deg):
        q.append(((2 * m + 1) * a * q[m] - m * b * b * q[m - 1]) / (m + 1))
    cols = []
    for m in range(deg + 1):
        jac = jacobi(deg - m, 2 * m + 1, 2 * y - 1)
        for n in range(deg + 1 - m):
            cols.append(q[m] * jac[n])
    return np.stack(cols, axis=-1)


def make_residual(n3, n21, n111, deg):
    nb = (deg + 1) * (deg + 2) // 2
    exact = np.zeros(nb)
    exact[0] = 0.5
    gx, gw = np.polynomial.legendre.leggauss(deg + 4)
    u, uw = 0.5 * (gx + 1), 0.5 * gw
    xs = np.outer(u, 1 - u).ravel()
    ys = np.outer(np.ones_like(u), u).ravel()
    ws = np.outer(uw, uw * (1 - u)).ravel()
    basis = dubiner(xs, ys, deg)
    norms = np.sqrt((ws[:, None] * basis * basis).sum(0))

    def residual(p):
        lam, w = expand(p, n3, n21, n111)
        return (w @ dubiner(lam[:, 1], lam[:, 2], deg) - exact) / norms

    return residual


def polish(p, residual, iters=50):
    r = residual(p)
    mu = 1e-8
    for _ in range(iters):
        jac = np.empty((len(r), len(p)))
        for j in range(len(p)):
            q = p.copy()
            q[j] += 1e-7
            jac[:, j] = (residual(q) - r) / 1e-7
        a = np.vstack([jac, np.sqrt(mu) * np.eye(len(p))])
        step = np.linalg.lstsq(a, np.concatenate([-r, np.zeros(len(p))]), rcond=None)[0]
        q = p + step
        rq = residual(q)
        if np.linalg.norm(rq) < np.linalg.norm(r):
            p, r = q, rq
            mu = max(mu / 5, 1e-18)
        else:
            mu *= 5
            if mu > 1e4:
                break
    return p


def monomial_error(lam, w, deg):
    err = 0.0
    for a in range(deg + 1):
        for b in range(deg + 1 - a):
            exact = math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
            err = max(err, abs(np.sum(w * lam[:, 1] ** a * lam[:, 2] ** b) - exact))
    return err


def build_rule(npts, deg, structure, start):
    n3, n21, n111 = structure
    p = polish(np.array(start, dtype=np.float64), make_residual(n3, n21, n111, deg))
    lam, w = expand(p, n3, n21, n111)
    err = monomial_error(lam, w, deg)
    if not (len(w) == npts and err < 1e-15 and np.all(lam > 1e-9) and np.all(w > 0)):
        raise RuntimeError(f"rule {npts} failed: err={err}")
    return lam, w, err


def main():
    out = sys.stdout
    out.write("// Generated by gen_simplex_rules.py: fully symmetric triangle rules on the\n")
    out.write("// reference triangle (0,0),(1,0),(0,1); weights sum to 1/2.\n")
    for npts, deg, structure, start in RULES:
        lam, w, err = build_rule(npts, deg, structure, start)
        name = f"kSimplexRule{npts}"
        out.write(f"// npoints={npts} degree={deg} max monomial moment error={err:.1e}\n")
        out.write(f"static const double {name}Points[{2 * npts}] = {{\n")
        for i in range(npts):
            out.write(f"    {float(lam[i, 1])!r}, {float(lam[i, 2])!r},\n")
        out.write("};\n")
        out.write(f"static const double {name}Weights[{npts}] = {{\n")
        for i in range(npts):
            out.write(f"    {float(w[i])!r},\n")
        out.write("};\n")
    out.write("static const SimplexRuleEntry kSimplexRules[] = {\n")
    for npts, deg, *_ in RULES:
        out.write(f"    {{{npts}, {deg}, kSimplexRule{npts}Points, kSimplexRule{npts}Weights}},\n")
    out.write("};\n")


if __name__ == "__main__":
    main()
