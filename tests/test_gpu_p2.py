"""Degree-2 Lagrange spaces (P2 and DP2, alone and paired with DP0 / P1) on the GPU
against the FP64 oracle, relative Frobenius error <= 1e-12.

These spaces go through the warp-per-cell-pair kernel (generic.cu) for the singular part
and for the regular part of every pairing but Laplace single / double / adjoint double
layer on P2 x P2, which the tiled kernel of regular.cu assembles.  The oracle's degree-2
basis is pinned to its P1 matrices, and those to the bempp-cl goldens, by
tests/test_oracle_golden.py (the P2 matrix restricted to the P1 subspace is the P1
matrix).
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

from test_gpu_parity import FP64_TOL, OPS, gpu_assemble, oracle_assemble, rel_err

pytestmark = pytest.mark.gpu

P2, DP2, P1, DP0 = (2, True), (2, False), (1, True), (0, False)


@pytest.fixture(scope="module")
def grid():
    pts, cells = shapes.icosphere(1)
    return Grid(shapes.radial_perturbation(pts, seed=17), cells)


CASES = [(kernel, op) for kernel in ("laplace", "helmholtz")
         for op in ("single_layer", "double_layer", "adjoint_double_layer", "hypersingular")]


@pytest.mark.parametrize("kernel,op", CASES)
@pytest.mark.parametrize("sp", [P2, DP2])
def test_degree2_matches_oracle(grid, kernel, op, sp):
    a = gpu_assemble(grid, kernel, op, 2.5, test=sp, trial=sp)
    o = oracle_assemble(grid, kernel, op, 2.5, test=sp, trial=sp)
    assert a.shape == o.shape
    assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("kernel,op,test,trial", [
    ("laplace", "double_layer", P2, P1),
    ("laplace", "hypersingular", P1, P2),
    ("helmholtz", "single_layer", P2, DP0),
    ("helmholtz", "adjoint_double_layer", DP0, P2),
    ("laplace", "single_layer", DP2, P1),
])
def test_degree2_paired_with_other_spaces(grid, kernel, op, test, trial):
    a = gpu_assemble(grid, kernel, op, 3.0, test=test, trial=trial)
    o = oracle_assemble(grid, kernel, op, 3.0, test=test, trial=trial)
    assert rel_err(a, o) <= FP64_TOL


def test_degree2_one_space_object_and_rules(grid):
    """One space object on both sides (the symmetric operators' launch) and other rules."""
    for q, order in ((3, 3), (7, 5)):
        a = gpu_assemble(grid, "helmholtz", "hypersingular", 4.0, test=P2, trial=P2, q=q,
                         order=order, one_space=True)
        o = oracle_assemble(grid, "helmholtz", "hypersingular", 4.0, test=P2, trial=P2, q=q,
                            order=order)
        assert rel_err(a, o) <= FP64_TOL


@pytest.mark.parametrize("op", ["single_layer", "double_layer", "adjoint_double_layer"])
def test_degree2_tiled_kernel_on_several_tiles(op):
    """Laplace P2 x P2 (single, double, adjoint double layer) goes through the tiled
    kernel (6 x 6 blocks per cell pair, per-tile DOF accumulation): 320 cells (10 tiles),
    one space object (the single layer then computes the tile pairs tx >= sy only)."""
    pts, cells = shapes.icosphere(2)
    g = Grid(shapes.radial_perturbation(pts, seed=23), cells)
    a = gpu_assemble(g, "laplace", op, test=P2, trial=P2, one_space=True)
    o = oracle_assemble(g, "laplace", op, test=P2, trial=P2)
    assert rel_err(a, o) <= FP64_TOL


def test_degree2_mixed_precision_option_gives_fp64(grid):
    """The precision option does not apply to degree-2 spaces: they are integrated in
    FP64."""
    a = gpu_assemble(grid, "helmholtz", "double_layer", 5.0, test=P2, trial=P2,
                     precision=Precision.Mixed)
    o = oracle_assemble(grid, "helmholtz", "double_layer", 5.0, test=P2, trial=P2)
    assert rel_err(a, o) <= FP64_TOL


def test_degree2_host_path_in_chunks_and_csr():
    """1,280 cells (2,562 P2 DOFs, 105 MB complex128): the host-memory path assembles it
    in chunks of trial cells with the singular pairs of each chunk; the singular part as
    CSR matches the oracle's."""
    import torch

    pts, cells = shapes.icosphere(3)
    g = Grid(shapes.radial_perturbation(pts, seed=5), cells)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    sp = function_space(g, create_family(Family.Lagrange, 2))
    a = create_helmholtz_assembler(OperatorType.SingleLayer, 3.0, opts)
    host = a.assemble(sp, sp)
    n = sp.global_size
    dev = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    a.assemble_into_device(sp, sp, dev, torch.cuda.current_stream().cuda_stream, check=True)
    dev = dev.cpu().numpy().T
    assert rel_err(host, dev) <= 1e-13
    rows = np.random.default_rng(2).choice(n, size=24, replace=False)
    from oracle import oracle

    dofs, _ = oracle.cell_dofs(g.points, g.cells, 2, True)
    tcells = np.flatnonzero(np.isin(dofs, rows).any(axis=1))
    o = oracle_assemble(g, "helmholtz", "single_layer", 3.0, test=P2, trial=P2,
                        test_subset=tcells)
    assert rel_err(host[rows], o[rows]) <= FP64_TOL
    csr = create_laplace_assembler(OperatorType.Hypersingular, opts).assemble_singular(sp, sp)
    os_ = oracle_assemble(g, "laplace", "hypersingular", test=P2, trial=P2, parts=2)
    assert rel_err(csr.toarray(), os_) <= FP64_TOL


@pytest.mark.parametrize("kernel,op", [("laplace", "single_layer"),
                                       ("helmholtz", "double_layer")])
def test_degree2_potential_matches_oracle(grid, kernel, op):
    from bempp.assembly.potential import (create_helmholtz_potential_assembler,
                                          create_laplace_potential_assembler)
    from oracle import potential

    rng = np.random.default_rng(4)
    x = rng.standard_normal((40, 3))
    x *= 2.0 / np.linalg.norm(x, axis=1, keepdims=True)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    sp = function_space(grid, create_family(Family.Lagrange, 2))
    if kernel == "laplace":
        p = create_laplace_potential_assembler(OPS[op], opts).assemble(sp, x)
    else:
        p = create_helmholtz_potential_assembler(OPS[op], 2.0, opts).assemble(sp, x)
    o = potential.potential(x, grid.points, grid.cells, kernel, op, k=2.0, degree=2,
                            continuous=True, q_regular=6)
    assert rel_err(p, o) <= FP64_TOL
