"""Quadrilateral grids on the GPU against the FP64 oracle (oracle/oracle_quad.cpp),
relative Frobenius error <= 1e-12: DP0, Q1 and DQ1 spaces, every operator of both
kernels, the regular part (Gauss tensor rules on both cells) and the singular part (the
49 quadrilateral Duffy configurations), dense and CSR, device and host memory.

The oracle's quadrilateral rules are checked by their own invariants (the closed-form
Coulomb energy of a square, edge / vertex splits, polynomial exactness) in
tests/test_oracle_golden.py, and the product's rules equal the oracle's point for point
(tests/test_quad_host.py)."""

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

from test_gpu_parity import FP64_TOL, OPS, rel_err

pytestmark = pytest.mark.gpu

Q = ReferenceCellType.Quadrilateral
DP0, Q1, DQ1 = (0, False), (1, True), (1, False)


def perturbed_cube(n, seed=3):
    pts, cells = shapes.cube_quads(n)
    rng = np.random.default_rng(seed)
    return pts * (1 + 0.04 * rng.standard_normal((len(pts), 1))), cells


@pytest.fixture(scope="module")
def cube():
    return Grid(*perturbed_cube(3))


@pytest.fixture(scope="module")
def screen():
    return Grid(*shapes.screen_quads(4))


def quad_options(q=16, order=4, precision=Precision.FP64):
    opts = BoundaryAssemblerOptions()
    if q is not None:
        opts.set_regular_quadrature_degree(Q, q)
    if order is not None:
        opts.set_singular_quadrature_degree(Q, Q, order)
    opts.set_precision(precision)
    return opts


def space(grid, sp):
    deg, cont = sp
    return function_space(grid, create_family(
        Family.Lagrange, deg, Continuity.Standard if cont else Continuity.Discontinuous))


def assembler(kernel, op, k, opts, dtype=None):
    if kernel == "laplace":
        return create_laplace_assembler(OPS[op], opts, dtype or np.float64)
    return create_helmholtz_assembler(OPS[op], k, opts, dtype or np.complex128)


def gpu_assemble(grid, kernel, op, k=0.0, test=DP0, trial=DP0, q=16, order=4, **kw):
    ts, ss = space(grid, test), space(grid, trial)
    return assembler(kernel, op, k, quad_options(q, order, **kw)).assemble(ss, ts)


def oracle_quad(grid, kernel, op, k=0.0, test=DP0, trial=DP0, q=16, order=4, parts=3):
    return oracle.quad_assemble(grid.points, grid.cells.astype(np.int64), kernel, op, k=k,
                                test_degree=test[0], test_continuous=test[1],
                                trial_degree=trial[0], trial_continuous=trial[1],
                                q_regular=q, q_singular=order, parts=parts)


CASES = [(kernel, op) for kernel in ("laplace", "helmholtz")
         for op in ("single_layer", "double_layer", "adjoint_double_layer", "hypersingular")]


@pytest.mark.parametrize("kernel,op", CASES)
@pytest.mark.parametrize("sp", [DP0, Q1, DQ1])
def test_quad_matches_oracle(cube, kernel, op, sp):
    if op == "hypersingular" and sp == DP0:
        pytest.skip("the hypersingular operator of piecewise constants is zero")
    a = gpu_assemble(cube, kernel, op, 2.0, test=sp, trial=sp)
    o = oracle_quad(cube, kernel, op, 2.0, test=sp, trial=sp)
    assert a.shape == o.shape
    assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("kernel,op,test,trial", [
    ("laplace", "double_layer", Q1, DP0),
    ("helmholtz", "single_layer", DP0, Q1),
    ("helmholtz", "hypersingular", Q1, DQ1),
    ("laplace", "adjoint_double_layer", DQ1, Q1),
])
def test_quad_mixed_spaces(cube, kernel, op, test, trial):
    a = gpu_assemble(cube, kernel, op, 1.5, test=test, trial=trial)
    o = oracle_quad(cube, kernel, op, 1.5, test=test, trial=trial)
    assert rel_err(a, o) <= FP64_TOL


def test_quad_open_screen_and_default_rules(screen):
    """The open screen of the reference's quadrilateral cases, with the default options
    (37 regular points: the 7 x 7 Gauss rule; Duffy order 4)."""
    opts = BoundaryAssemblerOptions()
    for kernel, op, sp in (("laplace", "single_layer", DP0), ("helmholtz", "hypersingular", Q1)):
        ts = space(screen, sp)
        a = assembler(kernel, op, 3.0, opts).assemble(ts, ts)
        o = oracle_quad(screen, kernel, op, 3.0, test=sp, trial=sp, q=37, order=4)
        assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("q,order", [(1, 2), (9, 3), (36, 6), (100, 5)])
def test_quad_other_rules(cube, q, order):
    a = gpu_assemble(cube, "helmholtz", "double_layer", 2.5, test=Q1, trial=Q1, q=q, order=order)
    o = oracle_quad(cube, "helmholtz", "double_layer", 2.5, test=Q1, trial=Q1, q=q, order=order)
    assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("kernel,op,sp", [("laplace", "hypersingular", Q1),
                                          ("laplace", "single_layer", DP0),
                                          ("helmholtz", "single_layer", DQ1),
                                          ("helmholtz", "hypersingular", Q1)])
def test_quad_one_space_object(cube, kernel, op, sp):
    """One space object on both sides of a symmetric operator: only the regular pairs with
    test cell >= trial cell are integrated, each also added at the transposed entries."""
    s = space(cube, sp)
    a = assembler(kernel, op, 2.0, quad_options()).assemble(s, s)
    o = oracle_quad(cube, kernel, op, 2.0, test=sp, trial=sp)
    assert rel_err(a, o) <= FP64_TOL


def test_quad_two_grids_have_no_singular_part():
    """Test and trial on two disjoint cubes: every pair is regular."""
    pts, cells = perturbed_cube(2)
    g1 = Grid(pts, cells)
    g2 = Grid(pts * 0.7 + np.array([3.0, 0.5, -0.2]), cells)
    ts, ss = space(g1, Q1), space(g2, DP0)
    a = assembler("helmholtz", "double_layer", 2.0, quad_options()).assemble(ss, ts)
    # the oracle on the union: the off-diagonal block is the two-grid matrix
    upts = np.vstack([g1.points, g2.points])
    ucells = np.vstack([cells, cells + len(pts)]).astype(np.int64)
    full_t, nt = oracle.quad_cell_dofs(upts, ucells, 1, True)
    o = oracle.quad_assemble(upts, ucells, "helmholtz", "double_layer", k=2.0, test_degree=1,
                             test_continuous=True, trial_degree=0, q_regular=16, q_singular=4)
    t_dofs = np.unique(full_t[:len(cells)])
    assert rel_err(a, o[np.ix_(t_dofs, np.arange(len(cells), 2 * len(cells)))]) <= FP64_TOL


def test_quad_device_memory_and_single_precision(cube):
    import torch

    sp = space(cube, Q1)
    a = assembler("helmholtz", "single_layer", 2.0, quad_options())
    n = sp.global_size
    dev = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    a.assemble_into_device(sp, sp, dev, torch.cuda.current_stream().cuda_stream, check=True)
    o = oracle_quad(cube, "helmholtz", "single_layer", 2.0, test=Q1, trial=Q1)
    assert rel_err(dev.cpu().numpy().T, o) <= FP64_TOL
    a32 = assembler("helmholtz", "single_layer", 2.0, quad_options(), np.complex64)
    sp32 = function_space(cube, create_family(Family.Lagrange, 1, dtype=np.float32))
    m32 = a32.assemble(sp32, sp32)
    assert m32.dtype == np.complex64
    assert rel_err(m32, o) <= 1e-6


def test_quad_singular_part_as_csr(cube):
    sp = space(cube, DQ1)
    csr = assembler("helmholtz", "adjoint_double_layer", 2.0, quad_options()).assemble_singular(
        sp, sp)
    o = oracle_quad(cube, "helmholtz", "adjoint_double_layer", 2.0, test=DQ1, trial=DQ1, parts=2)
    assert rel_err(csr.toarray(), o) <= FP64_TOL


def test_quad_mixed_precision_option_gives_fp64(cube):
    a = gpu_assemble(cube, "helmholtz", "single_layer", 4.0, test=DP0, trial=DP0,
                     precision=Precision.Mixed)
    o = oracle_quad(cube, "helmholtz", "single_layer", 4.0)
    assert rel_err(a, o) <= FP64_TOL


def test_quad_unsupported_uses_are_reported(cube):
    from bempp.assembly.potential import create_laplace_potential_assembler

    tri = Grid(*shapes.icosphere(0))
    with pytest.raises(Exception, match="triangle grid and a quadrilateral"):
        assembler("laplace", "single_layer", 0.0, quad_options()).assemble(
            space(cube, DP0), space(tri, DP0))
    with pytest.raises(Exception, match="quadrilateral"):
        create_laplace_potential_assembler(OperatorType.SingleLayer, quad_options()).assemble(
            space(cube, DP0), np.array([[3.0, 0.0, 0.0]]))
