"""C-ABI library and host logic, on the CPU (no kernel launches).

- the library loads and exports every function include/bempp_b200.h declares;
- options behave as bempp-rs's (python/test/test_boundary_assembler.py:10-43);
- function spaces have bempp-rs's sizes and DOF numbering (python/test/
  test_function_space.py, src/function.rs:365-445), checked against the oracle;
- the product's quadrature rules equal the oracle's, and are exact where they must be;
- the singular pair list is every ordered vertex-sharing pair exactly once;
- invalid input is reported, not crashed on.
"""

import ctypes
import os
import re

import numpy as np
import pytest

from bempp import _lib, shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,
                                     create_helmholtz_assembler, create_laplace_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid
from ndgrid.shapes import regular_sphere
from oracle import oracle

ffi, lib = _lib.ffi, _lib.lib


def declared_functions():
    text = open(_lib.HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)) -
                  {"if", "sizeof", "defined"})


def test_library_exports_every_declared_symbol():
    so = ctypes.CDLL(_lib.LIBRARY)
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(so, n)]
    assert missing == []


def test_reference_symbol_names_present():
    """The names the reference's Python binding calls (python/bempp/**)."""
    so = ctypes.CDLL(_lib.LIBRARY)
    for n in ["boundary_assembler_options_new", "boundary_assembler_options_t_free",
              "boundary_assembler_options_set_regular_quadrature_degree",
              "boundary_assembler_options_get_regular_quadrature_degree",
              "boundary_assembler_options_has_regular_quadrature_degree",
              "boundary_assembler_options_set_singular_quadrature_degree",
              "boundary_assembler_options_get_singular_quadrature_degree",
              "boundary_assembler_options_has_singular_quadrature_degree",
              "boundary_assembler_options_set_batch_size",
              "boundary_assembler_options_get_batch_size", "laplace_boundary_assembler_new",
              "helmholtz_boundary_assembler_new", "boundary_assembler_t_free",
              "boundary_assembler_dtype", "boundary_assembler_assemble",
              "boundary_assembler_assemble_singular", "boundary_assembler_assemble_into_memory",
              "matrix_shape0", "matrix_shape1", "matrix_dense_data", "matrix_dense_data_copy",
              "matrix_csr_data_size", "matrix_csr_data", "matrix_csr_data_copy",
              "matrix_csr_indices_size", "matrix_csr_indices", "matrix_csr_indices_copy",
              "matrix_csr_indptr_size", "matrix_csr_indptr", "matrix_csr_indptr_copy",
              "matrix_t_free", "function_space", "space_t_free", "space_local_space",
              "space_is_serial", "space_get_local_dof_numbers_size",
              "space_get_local_dof_numbers", "space_local_size", "space_global_size",
              "space_has_cell_dofs", "space_cell_dofs_size", "space_cell_dofs",
              "space_global_dof_index", "space_is_owned", "space_dtype",
              "space_ownership_process", "space_ownership_index",
              "single_element_grid_borrowed_create_bempp", "grid_t_free_bempp",
              "create_lagrange_family_bempp", "element_family_t_free_bempp"]:
        assert hasattr(so, n), n


@pytest.mark.parametrize("otype", [OperatorType.SingleLayer, OperatorType.DoubleLayer,
                                   OperatorType.AdjointDoubleLayer, OperatorType.Hypersingular])
def test_create_assembler(otype):
    """python/test/test_boundary_assembler.py:10-43, with the operator under test."""
    o = BoundaryAssemblerOptions()
    assert o.regular_quadrature_degree(ReferenceCellType.Triangle) == 37
    o.set_regular_quadrature_degree(ReferenceCellType.Triangle, 3)
    assert o.regular_quadrature_degree(ReferenceCellType.Triangle) == 3
    with pytest.raises(ValueError):
        o.set_regular_quadrature_degree(ReferenceCellType.Interval, 3)
    with pytest.raises(ValueError):
        o.regular_quadrature_degree(ReferenceCellType.Interval)
    tri = ReferenceCellType.Triangle
    assert o.singular_quadrature_degree(tri, tri) == 4
    o.set_singular_quadrature_degree(tri, tri, 3)
    assert o.singular_quadrature_degree(tri, tri) == 3
    with pytest.raises(ValueError):
        o.set_singular_quadrature_degree(ReferenceCellType.Interval, ReferenceCellType.Interval, 3)
    assert o.batch_size() == 128
    o.set_batch_size(4)
    assert o.batch_size() == 4
    a = create_laplace_assembler(otype, o)
    assert a.dtype == np.float64
    with pytest.raises(ValueError):
        o.set_batch_size(8)  # read-only once used
    h = create_helmholtz_assembler(otype, 2.0, BoundaryAssemblerOptions())
    assert h.dtype == np.complex128
    h32 = create_helmholtz_assembler(otype, 2.0, BoundaryAssemblerOptions(), np.complex64)
    assert h32.dtype == np.complex64


def test_invalid_operator_and_dtype_are_reported():
    o = BoundaryAssemblerOptions()
    with pytest.raises(ValueError):
        create_laplace_assembler(OperatorType.ElectricField, o)
    with pytest.raises(ValueError):
        create_laplace_assembler(OperatorType.SingleLayer, BoundaryAssemblerOptions(),
                                 np.complex128)
    assert lib.create_raviart_thomas_family_bempp(0, 0, lib.DType_F64) == ffi.NULL
    assert "not supported" in _lib.last_error()
    pts = np.zeros((3, 3))
    cells = np.array([[0, 1, 7]], dtype=np.uintp)
    g = lib.bempp_grid_from_points_cells(ffi.cast("void*", pts.ctypes.data), 3, lib.DType_F64,
                                         ffi.cast("size_t*", cells.ctypes.data), 1)
    assert g == ffi.NULL and "out of range" in _lib.last_error()


@pytest.mark.parametrize("level", range(4))
def test_space_sizes(level):
    """python/test/test_function_space.py:8-41 (DP0 and P1)."""
    grid = regular_sphere(level)
    dp0 = function_space(grid, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    assert dp0.local_size == dp0.global_size == grid.entity_count(ReferenceCellType.Triangle)
    assert dp0.is_serial
    p1 = function_space(grid, create_family(Family.Lagrange, 1))
    assert p1.local_size == p1.global_size == grid.entity_count(ReferenceCellType.Point)
    dp1 = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Discontinuous))
    assert dp1.global_size == 3 * grid.entity_count(ReferenceCellType.Triangle)


@pytest.mark.parametrize("mesh", ["octa2", "ico2"])
@pytest.mark.parametrize("degree,cont", [(0, False), (1, True), (1, False)])
def test_dof_numbering_matches_oracle(mesh, degree, cont):
    pts, cells = shapes.regular_sphere(2) if mesh == "octa2" else shapes.icosphere(2)
    grid = Grid(pts, cells)
    sp = function_space(grid, create_family(
        Family.Lagrange, degree, Continuity.Standard if cont else Continuity.Discontinuous))
    ref, n = oracle.cell_dofs(pts, cells, degree, cont)
    assert sp.global_size == n
    ours = np.array([sp.cell_dofs(c) for c in range(len(cells))])
    assert np.array_equal(ours, ref)
    if degree == 1 and cont:
        # vertex DOFs: get_local_dof_numbers(0, v) is the DOF of vertex v
        for c in range(0, len(cells), 7):
            for i in range(3):
                assert sp.get_local_dof_numbers(0, int(cells[c, i])) == [ref[c, i]]


def test_octahedron_p1_numbering_is_identity():
    """On regular_sphere(0) first-visit numbering equals vertex numbering, which is what
    the perm [0, 5, 2, 4, 3, 1] of tests/compare_to_bempp_cl.rs:102 relies on."""
    grid = regular_sphere(0)
    sp = function_space(grid, create_family(Family.Lagrange, 1))
    assert [sp.get_local_dof_numbers(0, v)[0] for v in range(6)] == list(range(6))


@pytest.mark.parametrize("npts", [1, 3, 6, 7, 12, 15, 16, 19, 25, 33, 37])
def test_regular_rules_equal_oracle_and_are_exact(npts):
    p = np.zeros(2 * npts)
    w = np.zeros(npts)
    assert lib.bempp_regular_rule(npts, ffi.cast("double*", p.ctypes.data),
                                  ffi.cast("double*", w.ctypes.data)) == npts
    op, ow = oracle.simplex_rule(npts)
    assert np.array_equal(p.reshape(-1, 2), op) and np.array_equal(w, ow)
    assert abs(w.sum() - 0.5) < 1e-15
    assert np.all(w > 0) and np.all(p > 0) and np.all(p.reshape(-1, 2).sum(1) < 1)
    assert lib.bempp_regular_rule(5, ffi.NULL, ffi.NULL) == 0


def _product_duffy(config, order):
    n = lib.bempp_singular_rule(config, order, ffi.NULL, ffi.NULL, ffi.NULL)
    tp, sp, w = np.zeros(2 * n), np.zeros(2 * n), np.zeros(n)
    lib.bempp_singular_rule(config, order, ffi.cast("double*", tp.ctypes.data),
                            ffi.cast("double*", sp.ctypes.data), ffi.cast("double*", w.ctypes.data))
    return tp.reshape(n, 2), sp.reshape(n, 2), w


@pytest.mark.parametrize("config", range(28))
def test_singular_rules_equal_oracle(config):
    for order in (1, 2, 4):
        tp, sp, w = _product_duffy(config, order)
        otp, osp, ow = oracle.duffy_rule(config, order)
        np.testing.assert_allclose(tp, otp, rtol=0, atol=1e-15)
        np.testing.assert_allclose(sp, osp, rtol=0, atol=1e-15)
        np.testing.assert_allclose(w, ow, rtol=0, atol=1e-15)
    # point counts of the Sauter-Schwab decompositions: 2, 5, 6 regions x n^4
    n = len(_product_duffy(config, 4)[2])
    assert n == (512 if config < 9 else (1280 if config < 27 else 1536))


def _exact_tri_tri_moment(a, b, c, d):
    """Integral over T x T of x0^a x1^b y0^c y1^d (T the reference triangle)."""
    from math import factorial as f

    return f(a) * f(b) / f(a + b + 2) * f(c) * f(d) / f(c + d + 2)


@pytest.mark.parametrize("config", [0, 4, 9, 14, 26, 27])
def test_singular_rules_integrate_polynomials(config):
    """A Duffy rule is a change of variables over T x T: it integrates smooth functions of
    (x, y) like a tensor rule, so low-degree monomials come out exact."""
    tp, sp, w = _product_duffy(config, 6)
    for (a, b, c, d) in [(0, 0, 0, 0), (1, 0, 0, 0), (0, 1, 1, 0), (2, 1, 0, 1), (1, 1, 1, 1),
                         (3, 0, 0, 2)]:
        val = np.sum(w * tp[:, 0] ** a * tp[:, 1] ** b * sp[:, 0] ** c * sp[:, 1] ** d)
        assert abs(val - _exact_tri_tri_moment(a, b, c, d)) < 1e-13


def test_singular_rules_share_the_common_entity():
    """Points of the shared vertex / edge coincide: for a vertex configuration (i, j) the
    physical distance of the rule's point pairs tends to zero only at the shared vertex,
    and the two reference points map to the same physical point when both cells are the
    same triangle with identified vertices."""
    ref = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    for config in range(27):
        tp, sp, _ = _product_duffy(config, 3)
        bt = np.column_stack([1 - tp.sum(1), tp])  # barycentric on the test cell
        bs = np.column_stack([1 - sp.sum(1), sp])
        # the barycentric weight of non-shared vertices vanishes together on both sides
        # as the Duffy variable xi -> 0: check the rule has points approaching the
        # common entity on both cells simultaneously
        assert np.min(bt.max(1)) > 0 and np.min(bs.max(1)) > 0
    del ref


def test_singular_pairs_are_every_vertex_sharing_pair_once():
    pts, cells = shapes.icosphere(2)
    grid = Grid(pts, cells)
    from bempp.function_space import recreate_grid

    g = recreate_grid(grid)
    try:
        n = lib.bempp_grid_singular_pairs(g, ffi.NULL, ffi.NULL, ffi.NULL)
        t = np.zeros(n, dtype=np.uintp)
        s = np.zeros(n, dtype=np.uintp)
        c = np.zeros(n, dtype=np.uintp)
        lib.bempp_grid_singular_pairs(g, ffi.cast("size_t*", t.ctypes.data),
                                      ffi.cast("size_t*", s.ctypes.data),
                                      ffi.cast("size_t*", c.ctypes.data))
    finally:
        lib.grid_t_free_bempp(g)
    got = set(zip(t.tolist(), s.tolist()))
    assert len(got) == n  # no duplicates
    expected = {}
    configs = ([[(i, j)] for i in range(3) for j in range(3)] +
               [p for te in ([1, 2], [0, 2], [0, 1]) for se in ([1, 2], [0, 2], [0, 1])
                for p in ([(te[0], se[0]), (te[1], se[1])], [(te[1], se[0]), (te[0], se[1])])] +
               [[(0, 0), (1, 1), (2, 2)]])
    for a in range(len(cells)):
        for b in range(len(cells)):
            shared = [(ti, si) for si in range(3) for ti in range(3)
                      if cells[a, ti] == cells[b, si]]
            if shared:
                expected[(a, b)] = configs.index(shared)
    assert got == set(expected)
    for ti, si, ci in zip(t, s, c):
        assert expected[(int(ti), int(si))] == int(ci)
    # grouped by configuration
    assert np.all(np.diff(c.astype(np.int64)) >= 0)


def test_header_parses_for_cffi():
    assert lib.DType_C64 == 3 and lib.OperatorType_Hypersingular == 3
    assert lib.ReferenceCellType_Triangle == 2 and lib.Continuity_Discontinuous == 1
    assert os.path.exists(_lib.LIBRARY)


@pytest.mark.parametrize("ntt,ty0,ty1", [
    (1, 0, 1), (5, 0, 5), (16, 0, 16), (17, 0, 17), (40, 0, 40), (640, 0, 640),
    (320, 0, 71), (320, 71, 142), (320, 300, 320), (321, 17, 50), (33, 32, 33),
])
def test_lower_tile_pair_order_is_a_bijection(ntt, ty0, ty1):
    """The tile-pair order of lower-triangle launches visits every pair (tx >= sy,
    sy in [ty0, ty1)) exactly once, in bands of 16 trial tiles."""
    n = lib.bempp_lower_tile_pairs(ntt, ty0, ty1, ffi.NULL, ffi.NULL, 0)
    rows = ty1 - ty0
    assert n == sum(ntt - s for s in range(ty0, ty1))
    tx = np.zeros(n, dtype=np.int32)
    sy = np.zeros(n, dtype=np.int32)
    assert lib.bempp_lower_tile_pairs(ntt, ty0, ty1, ffi.cast("int*", tx.ctypes.data),
                                      ffi.cast("int*", sy.ctypes.data), n) == n
    assert np.all(tx >= sy) and np.all(sy >= ty0) and np.all(sy < ty1) and np.all(tx < ntt)
    key = tx.astype(np.int64) * ntt + sy
    assert len(np.unique(key)) == n
    band = (sy - ty0) // 16
    assert np.all(np.diff(band) >= 0)  # bands in order
    if rows > 16:
        assert band.max() == (rows - 1) // 16


def test_lower_tile_pairs_rejects_bad_ranges():
    assert lib.bempp_lower_tile_pairs(10, 5, 4, ffi.NULL, ffi.NULL, 0) == -1
    assert lib.bempp_lower_tile_pairs(10, 0, 11, ffi.NULL, ffi.NULL, 0) == -1


def test_device_trim_with_nothing_cached():
    assert lib.bempp_device_trim() == 0


def test_potential_of_a_hypersingular_assembler_is_unsupported():
    """potential_assemble_into_memory checks the operator before touching the device."""
    pts, cells = shapes.regular_sphere(0)
    grid = Grid(pts, cells)
    sp = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Standard))
    a = create_laplace_assembler(OperatorType.Hypersingular, BoundaryAssemblerOptions())
    x = np.array([[2.0, 0.0, 0.0]])
    out = np.empty((1, sp.global_size))
    st = lib.potential_assemble_into_memory(a._rs_assembler, sp._rs_space,
                                            ffi.cast("double*", x.ctypes.data), 1,
                                            ffi.cast("void*", out.ctypes.data))
    assert st == lib.BemppStatus_Unsupported
    assert "single and double layer" in _lib.last_error()


# ------------------------------------------------------------------ colouring ---
def _colouring_checks(grid, space, vertex_disjoint):
    """The checks of tests/test_space.rs:181-246: every cell in exactly one colour, and
    (continuous spaces) no two cells of one colour share a vertex."""
    colouring = space.cell_colouring()[ReferenceCellType.Triangle]
    cells = [c for group in colouring for c in group]
    assert sorted(cells) == list(range(len(grid.cells)))  # a partition
    if vertex_disjoint:
        cv = grid.cells if grid.cell_vertices is None else grid.cell_vertices
        for group in colouring:
            verts = cv[group].ravel()
            assert len(np.unique(verts)) == len(verts)
    return colouring


def test_colouring_p1():
    grid = regular_sphere(2)
    space = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Standard))
    colouring = _colouring_checks(grid, space, True)
    assert len(colouring) > 1


def test_colouring_dp0_is_one_colour():
    grid = regular_sphere(2)
    space = function_space(grid, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    assert len(_colouring_checks(grid, space, False)) == 1


@pytest.mark.parametrize("degree,cont", [(0, False), (1, True), (1, False)])
def test_colouring_matches_oracle(degree, cont):
    pts, cells = shapes.icosphere(2)
    grid = Grid(pts, cells)
    space = function_space(grid, create_family(
        Family.Lagrange, degree, Continuity.Standard if cont else Continuity.Discontinuous))
    colouring = space.cell_colouring()[ReferenceCellType.Triangle]
    ours = np.zeros(len(cells), dtype=np.int64)
    for c, group in enumerate(colouring):
        ours[group] = c
    ref, n = oracle.colouring(pts, cells, degree, cont)
    assert n == len(colouring)
    assert np.array_equal(ours, ref)


# ---------------------------------------------- ndgrid-shaped grid ingestion ---
def _seam_mesh(level=2):
    """An icosphere whose cells with an odd index refer to duplicated copies of their
    points (same coordinates, new point indices); the topology still joins each copy
    with its original vertex, as an ndgrid grid built with merged vertices would."""
    pts, cells = shapes.icosphere(level)
    pts = shapes.radial_perturbation(pts, seed=level)
    npts = len(pts)
    dup_cells = cells.copy()
    odd = np.arange(1, len(cells), 2)
    dup_cells[odd] += npts
    points = np.vstack([pts, pts])
    return points, dup_cells, cells, pts


def _pairs(g):
    n = lib.bempp_grid_singular_pairs(g, ffi.NULL, ffi.NULL, ffi.NULL)
    t = np.zeros(n, dtype=np.uintp)
    s = np.zeros(n, dtype=np.uintp)
    c = np.zeros(n, dtype=np.uintp)
    lib.bempp_grid_singular_pairs(g, ffi.cast("size_t*", t.ctypes.data),
                                  ffi.cast("size_t*", s.ctypes.data),
                                  ffi.cast("size_t*", c.ctypes.data))
    return set(zip(t.tolist(), s.tolist(), c.tolist()))


def test_ndgrid_topology_joins_duplicated_points():
    """single_element_grid_borrowed_create_bempp with ndgrid's connectivity arrays: the
    topology's vertices (not the point indices) decide the P1 DOFs, the colouring and the
    vertex-sharing pairs, so the seam mesh numbers exactly like the merged mesh."""
    from bempp.function_space import grid_handle

    points, dup_cells, cells, pts = _seam_mesh()
    seam = Grid(points, dup_cells, cell_vertices=cells)
    merged = Grid(pts, cells)
    plain = Grid(points, dup_cells)  # the same arrays without the topology
    p1 = create_family(Family.Lagrange, 1, Continuity.Standard)
    s_seam, s_merged, s_plain = (function_space(g, p1) for g in (seam, merged, plain))
    assert s_seam.global_size == s_merged.global_size == len(pts)
    assert s_plain.global_size > len(pts)  # without the topology every copy is a vertex
    ref, n = oracle.cell_dofs(pts, cells, 1, True)
    assert np.array_equal(np.array([s_seam.cell_dofs(c) for c in range(len(cells))]), ref)
    a = s_seam.cell_colouring()[ReferenceCellType.Triangle]
    b = s_merged.cell_colouring()[ReferenceCellType.Triangle]
    assert a == b
    assert _pairs(grid_handle(seam).ptr) == _pairs(grid_handle(merged).ptr)
    assert len(_pairs(grid_handle(plain).ptr)) < len(_pairs(grid_handle(merged).ptr))


def test_ndgrid_topology_with_renumbered_vertices():
    """A topology whose vertex ids are a permutation of the point indices changes nothing
    the assembly sees: DOFs (first visit) and vertex-sharing pairs are unchanged."""
    from bempp.function_space import grid_handle

    pts, cells = shapes.icosphere(2)
    perm = np.random.default_rng(3).permutation(len(pts))
    renum = Grid(pts, cells, cell_vertices=perm[cells])
    plain = Grid(pts, cells)
    p1 = create_family(Family.Lagrange, 1, Continuity.Standard)
    a, b = function_space(renum, p1), function_space(plain, p1)
    assert all(a.cell_dofs(c) == b.cell_dofs(c) for c in range(len(cells)))
    assert _pairs(grid_handle(renum).ptr) == _pairs(grid_handle(plain).ptr)
    # vertex DOFs are looked up by the topology's vertex id
    for c in range(0, len(cells), 11):
        for i in range(3):
            assert a.get_local_dof_numbers(0, int(perm[cells[c, i]])) == [b.cell_dofs(c)[i]]


def test_ndgrid_topology_is_validated():
    points, dup_cells, cells, pts = _seam_mesh(1)
    grid = Grid(points, dup_cells, cell_vertices=cells)
    t = grid.topology_arrays()
    # an edge list that disagrees with the cells' vertices is refused
    from bempp.function_space import _ndgrid_create

    t["edge_vertices"][0] = t["edge_vertices"][1]
    grid.topology_arrays = lambda: t
    g = _ndgrid_create(grid, np.ascontiguousarray(points), np.ascontiguousarray(dup_cells,
                                                                               dtype=np.uintp))
    assert g == ffi.NULL
    assert "disagrees" in _lib.last_error()
    # a cell -> vertex id beyond entity_counts[0]
    t2 = Grid(points, dup_cells, cell_vertices=cells).topology_arrays()
    t2["entity_counts"][0] = len(pts) - 1
    grid.topology_arrays = lambda: t2
    g = _ndgrid_create(grid, np.ascontiguousarray(points), np.ascontiguousarray(dup_cells,
                                                                               dtype=np.uintp))
    assert g == ffi.NULL
    assert "out of range" in _lib.last_error()


# ------------------------------------------------------------ degree-2 spaces ---
@pytest.mark.parametrize("level", range(3))
def test_space_sizes_p2(level):
    """python/test/test_function_space.py:31-41 and tests/test_space.rs (Lagrange 2): one
    DOF per vertex and per edge; DP2 has six per cell."""
    grid = regular_sphere(level)
    p2 = function_space(grid, create_family(Family.Lagrange, 2))
    assert p2.local_size == p2.global_size == (grid.entity_count(ReferenceCellType.Point) +
                                               grid.entity_count(ReferenceCellType.Interval))
    assert p2.is_serial
    dp2 = function_space(grid, create_family(Family.Lagrange, 2, Continuity.Discontinuous))
    assert dp2.global_size == 6 * grid.entity_count(ReferenceCellType.Triangle)


@pytest.mark.parametrize("cont", [True, False])
def test_p2_dof_numbering_matches_oracle(cont):
    pts, cells = shapes.icosphere(2)
    grid = Grid(pts, cells)
    sp = function_space(grid, create_family(
        Family.Lagrange, 2, Continuity.Standard if cont else Continuity.Discontinuous))
    ref, n = oracle.cell_dofs(pts, cells, 2, cont)
    assert sp.global_size == n
    assert np.array_equal(np.array([sp.cell_dofs(c) for c in range(len(cells))]), ref)
    if cont:
        # the edge DOFs: get_local_dof_numbers(1, e) is the DOF of edge e, and the cell's
        # local DOF 3 + i sits on its local edge i (opposite vertex i)
        seen = set()
        for c in range(len(cells)):
            for i in range(3):
                assert sp.get_local_dof_numbers(0, int(cells[c, i])) == [ref[c, i]]
            seen.update(int(d) for d in ref[c, 3:])
        edge_dofs = set()
        e = 0
        while True:
            d = sp.get_local_dof_numbers(1, e)
            if not d:
                break
            edge_dofs.update(d)
            e += 1
        assert edge_dofs == seen and e == len(seen)
        col = sp.cell_colouring()[ReferenceCellType.Triangle]
        ours = np.zeros(len(cells), dtype=np.int64)
        for k, group in enumerate(col):
            ours[group] = k
        refc, nc = oracle.colouring(pts, cells, 2, True)
        assert nc == len(col) and np.array_equal(ours, refc)


def test_p2_ndgrid_edge_numbering_is_kept():
    """Through ndgrid's arrays the edge DOFs hang on ndgrid's edges: the library keeps the
    given cell -> edge numbering, so entity (1, e) is ndgrid's edge e."""
    pts, cells = shapes.icosphere(1)
    grid = Grid(pts, cells, cell_vertices=cells)
    t = grid.topology_arrays()
    sp = function_space(grid, create_family(Family.Lagrange, 2))
    for c in range(len(cells)):
        dofs = sp.cell_dofs(c)
        for i in range(3):
            assert sp.get_local_dof_numbers(1, int(t["cell_edges"][c, i])) == [dofs[3 + i]]


def test_handles_alive_at_interpreter_exit_are_freed_quietly():
    """Options, assemblers, grids and spaces still referenced by module globals at exit
    are released by their finalizers while the library is still loaded."""
    import subprocess
    import sys

    pkg = os.path.dirname(os.path.dirname(_lib.__file__))
    # with torch loaded, the interpreter tears the modules down in an order in which a
    # __del__ running late finds cffi's function lookup already gone
    code = (
        "import numpy as np\n"
        "import torch\n"
        "from bempp import shapes\n"
        "from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,\n"
        "                                     create_laplace_assembler)\n"
        "from bempp.function_space import function_space\n"
        "from ndelement.ciarlet import Continuity, Family, create_family\n"
        "from ndgrid.grid import Grid\n"
        "opts = BoundaryAssemblerOptions()\n"
        "asm = create_laplace_assembler(OperatorType.SingleLayer, opts, np.float64)\n"
        "pts, cells = shapes.icosphere(1)\n"
        "grid = Grid(pts, cells)\n"
        "space = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Standard,\n"
        "                                           np.float64))\n"
        "print(space.global_size)\n")
    env = dict(os.environ, PYTHONPATH=pkg)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "42"
    assert "Exception ignored" not in r.stderr, r.stderr
