"""GPU parity: the CUDA assembler (through the C-ABI / Python binding) against the CPU
FP64 oracle on the same meshes, and against the bempp-cl golden matrices.

Tolerances: FP64 assembly must match the oracle to relative Frobenius error <= 1e-12
(same rules and formulas, only the summation order differs); the golden matrices are
checked entry-wise with the absolute epsilon of tests/compare_to_bempp_cl.rs.
"""

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType, Precision,
                                     create_helmholtz_assembler, create_laplace_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid
from oracle import oracle

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
OPS = {"single_layer": OperatorType.SingleLayer, "double_layer": OperatorType.DoubleLayer,
       "adjoint_double_layer": OperatorType.AdjointDoubleLayer,
       "hypersingular": OperatorType.Hypersingular}


def rel_err(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def gpu_assemble(grid, kernel, op, k=0.0, test=(0, False), trial=(0, False), q=6, order=4,
                 precision=Precision.FP64, dtype=None, one_space=False):
    """Dense matrix from the GPU assembler.  one_space: test and trial are the same space
    object, which lets symmetric operators (SL, HS) compute half of the tile pairs."""
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, q)
    opts.set_singular_quadrature_degree(ReferenceCellType.Triangle, ReferenceCellType.Triangle,
                                        order)
    opts.set_precision(precision)

    def space(deg, cont):
        return function_space(grid, create_family(
            Family.Lagrange, deg, Continuity.Standard if cont else Continuity.Discontinuous))

    ts = space(*test)
    ss = ts if one_space else space(*trial)
    if kernel == "laplace":
        a = create_laplace_assembler(OPS[op], opts, dtype or np.float64)
    else:
        a = create_helmholtz_assembler(OPS[op], k, opts, dtype or np.complex128)
    return a.assemble(ss, ts)


def oracle_assemble(grid, kernel, op, k=0.0, test=(0, False), trial=(0, False), q=6, order=4,
                    **kw):
    return oracle.assemble(grid.points, grid.cells.astype(np.int64), kernel, op, k=k,
                           test_degree=test[0], test_continuous=test[1], trial_degree=trial[0],
                           trial_continuous=trial[1], q_regular=q, q_singular=order, **kw)


@pytest.mark.parametrize("index", range(8))
def test_gpu_matches_bempp_cl_goldens(golden, index):
    case = golden["cases"][index]
    grid = Grid(*shapes.regular_sphere(0))
    sp = (case["degree"], case["continuous"])
    a = gpu_assemble(grid, case["kernel"], case["operator"], k=case["wavenumber"] or 0.0,
                     test=sp, trial=sp, q=37, order=4)
    m = np.array(case["matrix"])
    if m.ndim == 3:
        m = m[..., 0] + 1j * m[..., 1]
    ref = m[np.ix_(case["perm"], case["perm"])]
    assert np.abs(a.real - ref.real).max() <= case["epsilon"]
    assert np.abs(a.imag - ref.imag).max() <= case["epsilon"]
    o = oracle_assemble(grid, case["kernel"], case["operator"], k=case["wavenumber"] or 0.0,
                        test=sp, trial=sp, q=37, order=4)
    assert rel_err(a, o) <= FP64_TOL


SPACES = {"dp0": (0, False), "p1": (1, True), "dp1": (1, False)}
CASES = [
    ("laplace", "single_layer", "dp0", "dp0"),
    ("laplace", "double_layer", "dp0", "dp0"),
    ("laplace", "adjoint_double_layer", "dp0", "dp0"),
    ("laplace", "single_layer", "p1", "p1"),
    ("laplace", "double_layer", "p1", "p1"),
    ("laplace", "adjoint_double_layer", "p1", "p1"),
    ("laplace", "hypersingular", "p1", "p1"),
    ("laplace", "double_layer", "dp0", "p1"),
    ("laplace", "adjoint_double_layer", "p1", "dp0"),
    ("laplace", "single_layer", "dp1", "p1"),
    ("helmholtz", "single_layer", "dp0", "dp0"),
    ("helmholtz", "double_layer", "dp0", "dp0"),
    ("helmholtz", "adjoint_double_layer", "dp0", "dp0"),
    ("helmholtz", "double_layer", "p1", "p1"),
    ("helmholtz", "adjoint_double_layer", "p1", "p1"),
    ("helmholtz", "hypersingular", "p1", "p1"),
    ("helmholtz", "hypersingular", "dp0", "dp0"),
]


@pytest.mark.parametrize("kernel,op,test,trial", CASES)
@pytest.mark.parametrize("q", [6, 3])
def test_gpu_matches_oracle_small(kernel, op, test, trial, q):
    pts, cells = shapes.icosphere(1)
    pts = shapes.radial_perturbation(pts, seed=7)
    grid = Grid(pts, cells)
    k = 2.5
    a = gpu_assemble(grid, kernel, op, k, SPACES[test], SPACES[trial], q=q)
    o = oracle_assemble(grid, kernel, op, k, SPACES[test], SPACES[trial], q=q)
    assert a.shape == o.shape
    assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("kernel,op,sp", [("laplace", "single_layer", "dp0"),
                                          ("laplace", "hypersingular", "p1"),
                                          ("helmholtz", "double_layer", "p1")])
def test_gpu_matches_oracle_ico3(kernel, op, sp):
    """1,280-cell icosphere (the Laplace single-layer benchmark mesh), Q=6, order 4."""
    pts, cells = shapes.icosphere(3)
    grid = Grid(pts, cells)
    a = gpu_assemble(grid, kernel, op, 8.0, SPACES[sp], SPACES[sp])
    o = oracle_assemble(grid, kernel, op, 8.0, SPACES[sp], SPACES[sp])
    assert rel_err(a, o) <= FP64_TOL


def oracle_two_grids(g_test, g_trial, kernel, op, k=0.0, q=6):
    """DP0 x DP0 matrix between cells of two different grids from the oracle: assemble
    the union grid (g_test's cells, then g_trial's) for g_test's rows and keep the block
    of g_trial's columns.  Vertices are not shared between the two parts, so that block
    holds regular-rule entries only, as the assembler computes for two grid objects."""
    n1 = len(g_test.points)
    pts = np.vstack([g_test.points, g_trial.points])
    cells = np.vstack([g_test.cells.astype(np.int64), g_trial.cells.astype(np.int64) + n1])
    nc = len(g_test.cells)
    full = oracle_assemble(Grid(pts, cells), kernel, op, k, q=q, test_subset=np.arange(nc))
    return full[:nc, nc:]


@pytest.mark.parametrize("kernel,op,k", [("laplace", "single_layer", 0.0),
                                         ("laplace", "adjoint_double_layer", 0.0),
                                         ("helmholtz", "double_layer", 4.0)])
def test_different_grid_objects_have_no_singular_part(kernel, op, k):
    """Spaces on two grid objects: no pair is skipped and no Duffy rule is used, as
    equal_grids (pointer equality) in bempp-rs; the second sphere is shifted by less
    than its radius, so the regular rule also meets close and intersecting cell pairs."""
    pts, cells = shapes.icosphere(2)
    g1 = Grid(shapes.radial_perturbation(pts, seed=5), cells)
    g2 = Grid(shapes.radial_perturbation(pts, seed=6) + np.array([0.5, 0.2, 0.0]), cells)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    a = (create_laplace_assembler(OPS[op], opts) if kernel == "laplace"
         else create_helmholtz_assembler(OPS[op], k, opts))
    s1 = function_space(g1, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    s2 = function_space(g2, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    m = a.assemble(s2, s1)  # trial on g2, test on g1
    o = oracle_two_grids(g1, g2, kernel, op, k)
    assert m.shape == o.shape
    assert rel_err(m, o) <= FP64_TOL


def test_singular_csr_matches_dense():
    """python/test/test_boundary_assembler.py:45-68: every CSR singular entry equals the
    dense entry (discontinuous spaces on the octahedron)."""
    grid = Grid(*shapes.regular_sphere(0))
    for op in OPS.values():
        for td in (0, 1):
            for sd in (0, 1):
                ts = function_space(grid, create_family(Family.Lagrange, td, Continuity.Discontinuous))
                ss = function_space(grid, create_family(Family.Lagrange, sd, Continuity.Discontinuous))
                a = create_laplace_assembler(op)
                csr = a.assemble_singular(ss, ts).tocoo()
                dense = a.assemble(ss, ts)
                for i, j, v in zip(csr.row, csr.col, csr.data):
                    assert np.isclose(dense[i, j], v)


@pytest.mark.parametrize("kernel,op,k,sp", [
    ("laplace", "single_layer", 0.0, (0, False)),
    ("laplace", "single_layer", 0.0, (1, True)),
    ("laplace", "hypersingular", 0.0, (1, True)),
    ("helmholtz", "single_layer", 5.0, (0, False)),
    ("helmholtz", "hypersingular", 5.0, (1, True)),
    ("laplace", "double_layer", 0.0, (1, True)),
    ("laplace", "adjoint_double_layer", 0.0, (1, True)),
    ("laplace", "double_layer", 0.0, (1, False)),
    ("laplace", "adjoint_double_layer", 0.0, (1, False)),
    ("helmholtz", "double_layer", 5.0, (1, True)),
    ("helmholtz", "adjoint_double_layer", 5.0, (1, True)),
])
def test_one_space_symmetric_operators_match_oracle(kernel, op, k, sp):
    """Operators on one space object.  Single layer and hypersingular: only tile pairs
    (tx >= sy) are computed and the rest is mirrored.  The double layer and its adjoint
    on P1 / DP1: tile pairs (tx >= sy), each integrated in both orders from one kernel
    evaluation per point pair (Helmholtz: when the pair-referenced phase applies, as at
    k = 5 here).  The matrix matches the oracle, which computes every pair."""
    pts, cells = shapes.icosphere(3)
    grid = Grid(shapes.radial_perturbation(pts, seed=11), cells)
    a = gpu_assemble(grid, kernel, op, k, test=sp, trial=sp, one_space=True)
    o = oracle_assemble(grid, kernel, op, k, test=sp, trial=sp)
    err = rel_err(a, o)
    if err > FP64_TOL:  # where the entries differ, for the failure message
        bad = np.argwhere(np.abs(a - o) > 1e-9 * np.abs(o).max())
        tiles = sorted({(int(i) // 32, int(j) // 32) for i, j in bad})
        msg = (f"{len(bad)} entries differ; first {bad[:5].tolist()}; tile pairs {tiles[:20]}; "
               f"zeros in the result {int((a == 0).sum())}")
    else:
        msg = ""
    assert err <= FP64_TOL, msg



@pytest.mark.parametrize("op", ["double_layer", "adjoint_double_layer"])
@pytest.mark.parametrize("mesh", ["ico1", "open_cap"])
def test_paired_double_layer_on_ragged_tiles(op, mesh):
    """The paired launch (one P1 space object, Laplace DL / ADL) on meshes whose cell count
    is not a multiple of the 32-cell tile: the 80-cell icosphere (tiles of 32, 32, 16) and
    the 1,280-cell sphere with a polar cap removed (an open surface, last tile partial)."""
    pts, cells = shapes.icosphere(1 if mesh == "ico1" else 3)
    pts = shapes.radial_perturbation(pts, seed=31)
    if mesh == "open_cap":
        keep = pts[cells].mean(axis=1)[:, 2] < 0.8
        cells = cells[keep]
        used = np.unique(cells)
        remap = np.full(len(pts), -1)
        remap[used] = np.arange(len(used))
        pts, cells = pts[used], remap[cells]
        assert len(cells) % 32 != 0
    grid = Grid(pts, cells)
    a = gpu_assemble(grid, "laplace", op, test=(1, True), trial=(1, True), one_space=True)
    o = oracle_assemble(grid, "laplace", op, test=(1, True), trial=(1, True))
    assert rel_err(a, o) <= FP64_TOL


# ------------------------------------------------- singular part as CSR (row f1) ---
@pytest.mark.parametrize("kernel,op,k,sp", [
    ("laplace", "single_layer", 0.0, "dp0"),
    ("laplace", "double_layer", 0.0, "p1"),
    ("laplace", "adjoint_double_layer", 0.0, "dp1"),
    ("laplace", "hypersingular", 0.0, "p1"),
    ("helmholtz", "single_layer", 3.0, "p1"),
    ("helmholtz", "hypersingular", 3.0, "p1"),
])
def test_singular_csr_matches_oracle_singular_part(kernel, op, k, sp):
    """assemble_singular (src/boundary_assemblers.rs:121-155) against the oracle's
    singular part alone (parts=2): the same entries, summed over the pairs that share
    them, within the FP64 tolerance."""
    pts, cells = shapes.icosphere(2)
    grid = Grid(shapes.radial_perturbation(pts, seed=21), cells)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    a = (create_laplace_assembler(OPS[op], opts) if kernel == "laplace"
         else create_helmholtz_assembler(OPS[op], k, opts))
    fam = create_family(Family.Lagrange, SPACES[sp][0],
                        Continuity.Standard if SPACES[sp][1] else Continuity.Discontinuous)
    s = function_space(grid, fam)
    csr = a.assemble_singular(s, s)
    o = oracle_assemble(grid, kernel, op, k, SPACES[sp], SPACES[sp], parts=2)
    assert csr.shape == o.shape
    assert csr.nnz > 0
    assert rel_err(csr.toarray(), o) <= FP64_TOL


def test_singular_csr_of_a_negligible_part_is_empty():
    """src/boundary_assemblers.rs:130-145: when no singular entry exceeds 1e-10 in
    magnitude the result is an empty CSR matrix of the right shape (a sphere of radius
    1e-4: every entry is below 1e-10); spaces on two grid objects have no singular part."""
    pts, cells = shapes.icosphere(1)
    small = Grid(pts * 1e-4, cells)
    a = create_laplace_assembler(OperatorType.SingleLayer)
    s = function_space(small, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    csr = a.assemble_singular(s, s)
    assert csr.shape == (len(cells), len(cells)) and csr.nnz == 0
    assert np.all(csr.indptr == 0)
    dense = a.assemble(s, s)
    assert 0 < np.abs(dense).max() < 1e-10  # the entries exist, they are just negligible
    g1, g2 = Grid(pts, cells), Grid(pts + 3.0, cells)
    fam = create_family(Family.Lagrange, 1, Continuity.Standard)
    csr = a.assemble_singular(function_space(g2, fam), function_space(g1, fam))
    assert csr.nnz == 0 and csr.shape == (len(pts), len(pts))


# ------------------------------------------- ndgrid topology at the boundary (f2) ---
@pytest.mark.parametrize("kernel,op,sp", [("laplace", "single_layer", "dp0"),
                                          ("laplace", "hypersingular", "p1"),
                                          ("helmholtz", "double_layer", "p1")])
def test_seam_mesh_through_ndgrid_topology_matches_merged_mesh(kernel, op, sp):
    """Half of the cells refer to duplicated points; the ndgrid topology joins each copy
    with its original vertex.  The assembler must see the merged surface: singular pairs
    across the seam and shared P1 DOFs, i.e. the oracle's matrix of the merged mesh."""
    pts, cells = shapes.icosphere(2)
    pts = shapes.radial_perturbation(pts, seed=2)
    dup = cells.copy()
    dup[1::2] += len(pts)
    seam = Grid(np.vstack([pts, pts]), dup, cell_vertices=cells)
    a = gpu_assemble(seam, kernel, op, 4.0, SPACES[sp], SPACES[sp])
    o = oracle_assemble(Grid(pts, cells), kernel, op, 4.0, SPACES[sp], SPACES[sp])
    assert rel_err(a, o) <= FP64_TOL
