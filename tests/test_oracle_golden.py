"""The CPU oracle against bempp-rs's own known-answer tests.

tests/compare_to_bempp_cl.rs (bempp-rs) compares eight matrices assembled on the unit
octahedron with default options (37-point regular rule, order-4 Duffy rules) against
bempp-cl within an absolute epsilon (1e-3 or 1e-4, per test).  The same comparison,
entry by entry and with the same tolerance and DOF permutation, pins the oracle here.
"""

import numpy as np
import pytest

from bempp import shapes
from oracle import oracle


def _golden_matrix(case):
    m = np.array(case["matrix"])
    if m.ndim == 3:
        m = m[..., 0] + 1j * m[..., 1]
    p = case["perm"]
    return m[np.ix_(p, p)]


@pytest.mark.parametrize("index", range(8))
def test_oracle_matches_bempp_cl(golden, index):
    case = golden["cases"][index]
    pts, cells = shapes.regular_sphere(0)
    a = oracle.assemble(pts, cells, case["kernel"], case["operator"],
                        k=case["wavenumber"] or 0.0, test_degree=case["degree"],
                        test_continuous=case["continuous"], trial_degree=case["degree"],
                        trial_continuous=case["continuous"])
    ref = _golden_matrix(case)
    eps = case["epsilon"]  # absolute, as assert_relative_eq!(.., epsilon = eps)
    assert np.abs(a.real - ref.real).max() <= eps
    if np.iscomplexobj(ref):
        assert np.abs(a.imag - ref.imag).max() <= eps


def test_singular_part_is_subset_of_dense():
    """python/test/test_boundary_assembler.py:45-68: every singular entry equals the
    dense entry; here checked as dense = regular + singular on a refined sphere."""
    pts, cells = shapes.regular_sphere(1)
    for op in oracle.OPERATORS:
        deg = 1 if op == "hypersingular" else 0
        kw = dict(test_degree=deg, test_continuous=bool(deg), trial_degree=deg,
                  trial_continuous=bool(deg), q_regular=6)
        dense = oracle.assemble(pts, cells, "laplace", op, **kw)
        reg = oracle.assemble(pts, cells, "laplace", op, parts=1, **kw)
        sing = oracle.assemble(pts, cells, "laplace", op, parts=2, **kw)
        np.testing.assert_allclose(reg + sing, dense, rtol=0, atol=1e-15)
        assert np.count_nonzero(sing) > 0


@pytest.fixture(scope="module")
def golden_potentials():
    import json
    import os

    path = os.path.join(os.path.dirname(__file__), "golden", "bempp_cl_octahedron_potentials.json")
    with open(path) as f:
        return json.load(f)


@pytest.mark.parametrize("index", range(4))
def test_potential_oracle_matches_bempp_cl(golden_potentials, index):
    """The four potential-operator comparisons that tests/compare_to_bempp_cl.rs keeps
    commented out (lines 208-320): single and double layer potentials (Laplace, Helmholtz
    k = 3) of DP0 on the octahedron at three points, from_cl[dof][point] against
    matrix[point, dof], absolute epsilon 1e-3, default 37-point rule."""
    from oracle import potential

    case = golden_potentials["cases"][index]
    pts, cells = shapes.regular_sphere(0)
    p = potential.potential(case["points"], pts, cells, case["kernel"], case["operator"],
                            k=case["wavenumber"] or 0.0)
    ref = np.array(case["matrix"])
    if ref.ndim == 3:
        ref = ref[..., 0] + 1j * ref[..., 1]
    ref = ref.T  # [point, dof]
    assert p.shape == ref.shape
    assert np.abs(p.real - ref.real).max() <= case["epsilon"]
    if np.iscomplexobj(ref):
        assert np.abs(p.imag - ref.imag).max() <= case["epsilon"]


@pytest.mark.parametrize("kernel,op,k", [("laplace", "single_layer", 0.0),
                                         ("laplace", "double_layer", 0.0),
                                         ("laplace", "adjoint_double_layer", 0.0),
                                         ("laplace", "hypersingular", 0.0),
                                         ("helmholtz", "single_layer", 3.0),
                                         ("helmholtz", "hypersingular", 3.0)])
def test_oracle_p2_restricted_to_p1_is_the_p1_matrix(kernel, op, k):
    """The degree-2 Lagrange space contains the degree-1 one: phi_v(P1) = phi_v(P2) +
    (phi_e1 + phi_e2) / 2 over the two edges of the cell at v.  With that interpolation T,
    T^T A(P2) T must equal A(P1), whose values and derivatives the bempp-cl goldens pin
    (the hypersingular operator tests the P2 derivatives and the edge DOF order)."""
    pts, cells = shapes.icosphere(1)
    pts = shapes.radial_perturbation(pts, seed=3)
    d2, n2 = oracle.cell_dofs(pts, cells, 2, True)
    d1, n1 = oracle.cell_dofs(pts, cells, 1, True)
    T = np.zeros((n2, n1))
    for c in range(len(cells)):
        for i in range(3):
            T[d2[c, i], d1[c, i]] = 1.0
        for e in range(3):  # local edge e joins local vertices e+1, e+2 (mod 3)
            T[d2[c, 3 + e], d1[c, (e + 1) % 3]] = 0.5
            T[d2[c, 3 + e], d1[c, (e + 2) % 3]] = 0.5
    kw = dict(k=k, q_regular=6)
    a2 = oracle.assemble(pts, cells, kernel, op, test_degree=2, test_continuous=True,
                         trial_degree=2, trial_continuous=True, **kw)
    a1 = oracle.assemble(pts, cells, kernel, op, test_degree=1, test_continuous=True,
                         trial_degree=1, trial_continuous=True, **kw)
    r = T.T @ a2 @ T
    assert np.linalg.norm(r - a1) / np.linalg.norm(a1) <= 1e-13


def test_oracle_p2_potential_restricted_to_p1():
    from oracle import potential

    pts, cells = shapes.icosphere(1)
    d2, n2 = oracle.cell_dofs(pts, cells, 2, True)
    d1, n1 = oracle.cell_dofs(pts, cells, 1, True)
    T = np.zeros((n2, n1))
    for c in range(len(cells)):
        for i in range(3):
            T[d2[c, i], d1[c, i]] = 1.0
        for e in range(3):
            T[d2[c, 3 + e], d1[c, (e + 1) % 3]] = 0.5
            T[d2[c, 3 + e], d1[c, (e + 2) % 3]] = 0.5
    x = np.array([[2.0, 0.1, 0.0], [0.0, -1.7, 0.4], [0.3, 0.2, 2.5]])
    p2 = potential.potential(x, pts, cells, "helmholtz", "double_layer", k=2.0, degree=2,
                             continuous=True, q_regular=6)
    p1 = potential.potential(x, pts, cells, "helmholtz", "double_layer", k=2.0, degree=1,
                             continuous=True, q_regular=6)
    assert np.linalg.norm(p2 @ T - p1) / np.linalg.norm(p1) <= 1e-13


# ------------------------------------------------------------ quadrilateral rules ---
def _quad_configs():
    edges = [(0, 1), (0, 2), (1, 3), (2, 3)]
    out = [[(t, s)] for t in range(4) for s in range(4)]
    for te in range(4):
        for se in range(4):
            out.append([(edges[te][0], edges[se][0]), (edges[te][1], edges[se][1])])
            out.append([(edges[te][1], edges[se][0]), (edges[te][0], edges[se][1])])
    out.append([(0, 0), (1, 1), (2, 2), (3, 3)])
    return out


def test_quad_duffy_identical_rule_gives_the_coulomb_energy_of_a_square():
    """int_Q int_Q 1/|x - y| over the unit square = 4 ln(1 + sqrt 2) - (4/3)(sqrt 2 - 1)."""
    exact = 4 * np.log(1 + np.sqrt(2)) - 4 / 3 * (np.sqrt(2) - 1)
    tp, sp, w = oracle.quad_duffy_rule(48, 10)
    assert abs(np.sum(w / np.linalg.norm(tp - sp, axis=1)) - exact) <= 1e-12


def _bilinear(v, xi):
    s, t = xi[:, 0:1], xi[:, 1:2]
    return v[0] * (1 - s) * (1 - t) + v[1] * s * (1 - t) + v[2] * (1 - s) * t + v[3] * s * t


def _quad_pair_integral(x, y, order):
    pairs = [(ti, si) for si in range(4) for ti in range(4) if np.allclose(x[ti], y[si])]
    tp, sp, w = oracle.quad_duffy_rule(_quad_configs().index(pairs), order)
    return np.sum(w / np.linalg.norm(_bilinear(x, tp) - _bilinear(y, sp), axis=1))


def test_quad_duffy_edge_and_vertex_rules_split_the_coulomb_energy():
    """Two unit squares sharing an edge: E(2 x 1 rectangle) = 2 E(square) + 2 I_edge;
    four squares of a 2 x 2 square: 8 E = 4 E + 8 I_edge + 4 I_vertex.  Checked for every
    local numbering of the cells (each maps the shared entity by another symmetry)."""
    e = 4 * np.log(1 + np.sqrt(2)) - 4 / 3 * (np.sqrt(2) - 1)
    tp, sp, w = oracle.quad_duffy_rule(48, 16)
    d = tp - sp
    d[:, 0] *= 2.0
    e_rect = 4.0 * np.sum(w / np.linalg.norm(d, axis=1))  # the 2 x 1 rectangle
    i_edge = (e_rect - 2 * e) / 2
    i_vertex = e - 2 * i_edge
    a = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], float)
    b = a + np.array([1.0, 0.0, 0.0])
    c = a + np.array([1.0, 1.0, 0.0])
    # the eight numberings of a square's vertices that keep it a valid cell (D4)
    perms = [[0, 1, 2, 3], [1, 3, 0, 2], [3, 2, 1, 0], [2, 0, 3, 1],
             [1, 0, 3, 2], [0, 2, 1, 3], [2, 3, 0, 1], [3, 1, 2, 0]]
    for pa in perms:
        for pb in perms[::3]:
            assert abs(_quad_pair_integral(a[pa], b[pb], 10) - i_edge) <= 1e-12
            assert abs(_quad_pair_integral(a[pa], c[pb], 10) - i_vertex) <= 1e-12


@pytest.mark.parametrize("config", [0, 5, 15, 16, 23, 47, 48])
def test_quad_duffy_rules_integrate_polynomials(config):
    """The rules cover both squares exactly: products of monomials in the reference
    coordinates of the two cells integrate to the products of their 1-D moments."""
    tp, sp, w = oracle.quad_duffy_rule(config, 8)  # Gauss order 8: exact to degree 15 per axis
    assert abs(w.sum() - 1.0) <= 1e-13
    for a_, b_, c_, d_ in [(1, 0, 0, 0), (0, 1, 1, 0), (2, 1, 0, 3), (1, 1, 1, 1), (3, 0, 2, 2)]:
        f = tp[:, 0] ** a_ * tp[:, 1] ** b_ * sp[:, 0] ** c_ * sp[:, 1] ** d_
        exact = 1.0 / ((a_ + 1) * (b_ + 1) * (c_ + 1) * (d_ + 1))
        assert abs(np.sum(w * f) - exact) <= 1e-12


def test_quad_oracle_is_deterministic_across_threads():
    """Continuous spaces share DOFs between cells: the quadrilateral oracle's threads must
    not add into one entry at once (equal results for 1 and 8 threads, bit for bit)."""
    pts, cells = shapes.cube_quads(3)
    rng = np.random.default_rng(3)
    pts = pts * (1 + 0.04 * rng.standard_normal((len(pts), 1)))
    kw = dict(k=2.0, test_degree=1, test_continuous=True, trial_degree=1, trial_continuous=True)
    one = oracle.quad_assemble(pts, cells, "helmholtz", "adjoint_double_layer", nthreads=1, **kw)
    many = oracle.quad_assemble(pts, cells, "helmholtz", "adjoint_double_layer", nthreads=8, **kw)
    assert np.array_equal(one, many)
