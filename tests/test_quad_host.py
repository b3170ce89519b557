"""Quadrilateral grids through the C-ABI, on the CPU (no kernel launches): the product's
quadrilateral rules equal the oracle's, spaces number their DOFs as the oracle (and
bempp-rs's assign_dofs, src/function.rs:365-445) does, and the singular pair list is every
ordered vertex-sharing pair once with its configuration."""

import numpy as np
import pytest

from bempp import _lib, shapes
from bempp.function_space import function_space, recreate_grid
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid
from oracle import oracle

ffi, lib = _lib.ffi, _lib.lib

EDGES = [(0, 1), (0, 2), (1, 3), (2, 3)]


def quad_configs():
    out = [[(t, s)] for t in range(4) for s in range(4)]
    for te in range(4):
        for se in range(4):
            out.append([(EDGES[te][0], EDGES[se][0]), (EDGES[te][1], EDGES[se][1])])
            out.append([(EDGES[te][1], EDGES[se][0]), (EDGES[te][0], EDGES[se][1])])
    out.append([(0, 0), (1, 1), (2, 2), (3, 3)])
    return out


def product_quad_rule(config, order):
    n = lib.bempp_quadrilateral_singular_rule(config, order, ffi.NULL, ffi.NULL, ffi.NULL)
    tp, sp, w = np.zeros(2 * n), np.zeros(2 * n), np.zeros(n)
    lib.bempp_quadrilateral_singular_rule(config, order, ffi.cast("double*", tp.ctypes.data),
                                          ffi.cast("double*", sp.ctypes.data),
                                          ffi.cast("double*", w.ctypes.data))
    return tp.reshape(n, 2), sp.reshape(n, 2), w


@pytest.mark.parametrize("config", range(49))
def test_quad_singular_rules_equal_oracle(config):
    tp, sp, w = product_quad_rule(config, 4)
    otp, osp, ow = oracle.quad_duffy_rule(config, 4)
    assert len(w) == {1: 4, 2: 6, 4: 8}[len(quad_configs()[config])] * 4 ** 4
    np.testing.assert_allclose(tp, otp, rtol=0, atol=1e-15)
    np.testing.assert_allclose(sp, osp, rtol=0, atol=1e-15)
    np.testing.assert_allclose(w, ow, rtol=1e-14, atol=0)


@pytest.mark.parametrize("npts,n", [(1, 1), (4, 2), (16, 4), (17, 5), (37, 7), (256, 16)])
def test_quad_regular_rule_is_the_gauss_tensor_rule(npts, n):
    got = lib.bempp_quadrilateral_regular_rule(npts, ffi.NULL, ffi.NULL)
    assert got == n * n
    p, w = np.zeros(2 * n * n), np.zeros(n * n)
    lib.bempp_quadrilateral_regular_rule(npts, ffi.cast("double*", p.ctypes.data),
                                         ffi.cast("double*", w.ctypes.data))
    g, gw = np.polynomial.legendre.leggauss(n)
    g, gw = (g + 1) / 2, gw / 2
    np.testing.assert_allclose(p.reshape(-1, 2), np.array([[a, b] for a in g for b in g]),
                               atol=1e-15)
    np.testing.assert_allclose(w, np.outer(gw, gw).ravel(), rtol=1e-13)


def test_quad_regular_rule_above_the_limit_is_an_error():
    assert lib.bempp_quadrilateral_regular_rule(257, ffi.NULL, ffi.NULL) == 0


def perturbed_cube(n, seed=3):
    pts, cells = shapes.cube_quads(n)
    rng = np.random.default_rng(seed)
    return pts * (1 + 0.04 * rng.standard_normal((len(pts), 1))), cells


@pytest.mark.parametrize("degree,cont", [(0, Continuity.Discontinuous),
                                         (1, Continuity.Standard),
                                         (1, Continuity.Discontinuous)])
@pytest.mark.parametrize("mesh", ["cube", "screen"])
def test_quad_dof_numbering_matches_oracle(mesh, degree, cont):
    pts, cells = perturbed_cube(3) if mesh == "cube" else shapes.screen_quads(4)
    grid = Grid(pts, cells)
    assert grid.cell_type == ReferenceCellType.Quadrilateral
    space = function_space(grid, create_family(Family.Lagrange, degree, cont))
    ref, n = oracle.quad_cell_dofs(pts, cells, degree, cont == Continuity.Standard)
    assert space.global_size == n
    for c in range(len(cells)):
        assert space.cell_dofs(c) == ref[c].tolist()


def test_quad_space_sizes():
    pts, cells = shapes.cube_quads(4)
    grid = Grid(pts, cells)
    assert grid.entity_count(ReferenceCellType.Quadrilateral) == 96
    assert grid.entity_count(ReferenceCellType.Triangle) == 0
    assert grid.entity_count(ReferenceCellType.Point) == 98  # 6 n^2 + 2
    assert grid.entity_count(ReferenceCellType.Interval) == 192
    q1 = function_space(grid, create_family(Family.Lagrange, 1))
    dq1 = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Discontinuous))
    dp0 = function_space(grid, create_family(Family.Lagrange, 0))
    assert (q1.global_size, dq1.global_size, dp0.global_size) == (98, 384, 96)
    assert q1.element(ReferenceCellType.Quadrilateral).dim == 4


def test_quad_degree_two_is_unsupported():
    pts, cells = shapes.screen_quads(2)
    with pytest.raises(ValueError, match="quadrilateral"):
        function_space(Grid(pts, cells), create_family(Family.Lagrange, 2))


def test_quad_colouring_q1():
    pts, cells = shapes.screen_quads(4)
    space = function_space(Grid(pts, cells), create_family(Family.Lagrange, 1))
    groups = space.cell_colouring()[ReferenceCellType.Quadrilateral]
    assert sorted(c for g in groups for c in g) == list(range(len(cells)))
    for g in groups:  # no two cells of a colour share a vertex
        verts = cells[g].ravel()
        assert len(verts) == len(set(verts.tolist()))
    assert len(groups) == 4


@pytest.mark.parametrize("mesh", ["cube", "screen"])
def test_quad_singular_pairs_are_every_vertex_sharing_pair_once(mesh):
    pts, cells = perturbed_cube(2) if mesh == "cube" else shapes.screen_quads(3)
    g = recreate_grid(Grid(pts, cells))
    try:
        n = lib.bempp_grid_singular_pairs(g, ffi.NULL, ffi.NULL, ffi.NULL)
        t, s, c = (np.zeros(n, dtype=np.uintp) for _ in range(3))
        lib.bempp_grid_singular_pairs(g, ffi.cast("size_t*", t.ctypes.data),
                                      ffi.cast("size_t*", s.ctypes.data),
                                      ffi.cast("size_t*", c.ctypes.data))
    finally:
        lib.grid_t_free_bempp(g)
    configs = quad_configs()
    expected = {}
    for a in range(len(cells)):
        for b in range(len(cells)):
            shared = [(ti, si) for si in range(4) for ti in range(4)
                      if cells[a, ti] == cells[b, si]]
            if shared:
                expected[(a, b)] = configs.index(shared)
    got = dict(zip(zip(t.tolist(), s.tolist()), c.tolist()))
    assert len(got) == n
    assert got == expected
    assert np.all(np.diff(c.astype(np.int64)) >= 0)  # grouped by configuration


def test_quad_grid_with_triangle_connectivity_shape_is_rejected():
    """A quadrilateral grid whose cell -> vertex connectivity has 3 entries per cell."""
    pts, cells = shapes.screen_quads(2)
    cv = np.ascontiguousarray(cells, dtype=np.uintp)
    counts = np.array([len(pts), 12, len(cells)], dtype=np.uintp)
    d2 = ffi.new("size_t*[3]", [ffi.cast("size_t*", cv.ctypes.data), ffi.NULL, ffi.NULL])
    down = ffi.new("size_t**[3]", [ffi.new("size_t*[1]"), ffi.new("size_t*[2]"), d2])
    s2 = ffi.new("size_t[3]", [3, 4, 1])
    shape0 = ffi.new("size_t*[3]", [ffi.new("size_t[1]", [1]), ffi.new("size_t[2]", [2, 1]), s2])
    types = ffi.new("ReferenceCellType[3]", [lib.ReferenceCellType_Point,
                                             lib.ReferenceCellType_Interval,
                                             lib.ReferenceCellType_Quadrilateral])
    p = np.ascontiguousarray(pts)
    g = lib.single_element_grid_borrowed_create_bempp(
        2, ffi.NULL, ffi.NULL, types, ffi.cast("size_t*", counts.ctypes.data), down, shape0,
        ffi.NULL, ffi.NULL, ffi.cast("void*", p.ctypes.data), 3, len(pts), lib.DType_F64,
        ffi.cast("size_t*", cv.ctypes.data), 4, len(cells), 1)
    assert g == ffi.NULL
    assert b"4 entries per entity" in ffi.string(lib.bempp_last_error())
