"""The benchmark workloads at their own size against the FP64 oracle.

Each operator is assembled on the GPU at full size; the oracle computes complete rows
for a seeded subset of test DOFs (every cell holding one of those DOFs is a test cell of
the oracle's assembly, so those rows are complete), and the GPU's rows are compared with
them.  Tolerances: FP64 relative Frobenius error <= 1e-12 over the selected rows; mixed
precision <= 1e-6 (and > 1e-13: the FP32 path really ran).

* Laplace double layer, adjoint double layer and hypersingular, P1, on the
  20,480-triangle icosphere with a seeded radial perturbation (seed 20480);
* Helmholtz single layer (DP0) and double layer, adjoint double layer, hypersingular
  (P1) at k = 8 on the same mesh, FP64 and mixed;
* the batched Helmholtz single-layer sweep: 32 wavenumbers in [1, 20] on the stretched
  icospheres of 1,280, 5,120 and 20,480 triangles (seeds 1280, 5120, 20480), complex64:
  every (mesh, wavenumber) output.
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

OPS = {"single_layer": OperatorType.SingleLayer, "double_layer": OperatorType.DoubleLayer,
       "adjoint_double_layer": OperatorType.AdjointDoubleLayer,
       "hypersingular": OperatorType.Hypersingular}
NROWS = 32


@pytest.fixture(scope="module")
def ico5():
    pts, cells = shapes.icosphere(5)
    return Grid(shapes.radial_perturbation(pts, seed=20480), cells)


def row_subset(grid, degree, nrows, seed):
    """nrows test DOFs (seeded) and the cells that hold them."""
    dofs, n = oracle.cell_dofs(grid.points, grid.cells.astype(np.int64), degree,
                               degree == 1)
    rows = np.sort(np.random.default_rng(seed).choice(n, size=nrows, replace=False))
    cells = np.flatnonzero(np.isin(dofs, rows).any(axis=1))
    return rows, cells


def oracle_rows(grid, kernel, op, k, degree, rows, cells):
    o = oracle.assemble(grid.points, grid.cells.astype(np.int64), kernel, op, k=k,
                        test_degree=degree, test_continuous=degree == 1,
                        trial_degree=degree, trial_continuous=degree == 1, q_regular=6,
                        q_singular=4, test_subset=cells)
    return o[rows]


def gpu_rows(grid, kernel, op, k, degree, precision, rows):
    """Rows of the full-size matrix assembled into device memory (test and trial are one
    space object, as in the benchmark)."""
    import torch

    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    opts.set_precision(precision)
    fam = create_family(Family.Lagrange, degree,
                        Continuity.Standard if degree else Continuity.Discontinuous)
    sp = function_space(grid, fam)
    if kernel == "laplace":
        a = create_laplace_assembler(OPS[op], opts)
        dt = torch.float64
    else:
        a = create_helmholtz_assembler(OPS[op], k, opts)
        dt = torch.complex128
    n = sp.global_size
    out = torch.empty((n, n), dtype=dt, device="cuda")  # [trial, test]: column-major
    a.assemble_into_device(sp, sp, out, torch.cuda.current_stream().cuda_stream, check=True)
    r = out[:, torch.as_tensor(rows, device="cuda")].T.cpu().numpy()
    del out
    torch.cuda.empty_cache()
    return r


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


CASES = [
    ("laplace", "double_layer", 0.0, 1),
    ("laplace", "adjoint_double_layer", 0.0, 1),
    ("laplace", "hypersingular", 0.0, 1),
    ("helmholtz", "single_layer", 8.0, 0),
    ("helmholtz", "double_layer", 8.0, 1),
    ("helmholtz", "adjoint_double_layer", 8.0, 1),
    ("helmholtz", "hypersingular", 8.0, 1),
]


@pytest.mark.parametrize("kernel,op,k,degree", CASES)
def test_full_size_operator_rows_match_oracle(ico5, kernel, op, k, degree):
    rows, cells = row_subset(ico5, degree, NROWS, seed=100 + CASES.index((kernel, op, k, degree)))
    o = oracle_rows(ico5, kernel, op, k, degree, rows, cells)
    a64 = gpu_rows(ico5, kernel, op, k, degree, Precision.FP64, rows)
    assert rel(a64, o) <= 1e-12, (kernel, op, rel(a64, o))
    amx = gpu_rows(ico5, kernel, op, k, degree, Precision.Mixed, rows)
    e = rel(amx, o)
    assert 1e-13 < e <= 1e-6, (kernel, op, e)


def test_full_sweep_matches_oracle_rows():
    """Every output of the 32-wavenumber sweep over the three stretched meshes against
    oracle rows (64 rows on the two smaller meshes, 32 on the largest), complex64."""
    import torch

    from bempp.sweep import helmholtz_single_layer_sweep

    ks = np.linspace(1.0, 20.0, 32)
    grids = []
    for level, seed in ((3, 1280), (4, 5120), (5, 20480)):
        pts, cells = shapes.icosphere(level)
        grids.append(Grid(shapes.ellipsoidal_stretch(pts, seed), cells))
    outs = helmholtz_single_layer_sweep(grids, ks)
    torch.cuda.synchronize()
    worst = 0.0
    for g, out, nrows in zip(grids, outs, (64, 64, 32)):
        rows, cells = row_subset(g, 0, nrows, seed=len(g.cells))
        idx = torch.as_tensor(rows, device="cuda")
        for j, k in enumerate(ks):
            got = out[j][:, idx].T.to(torch.complex128).cpu().numpy()
            o = oracle_rows(g, "helmholtz", "single_layer", float(k), 0, rows, cells)
            e = rel(got, o)
            worst = max(worst, e)
            assert e <= 1e-6, (len(g.cells), k, e)
    del outs
    torch.cuda.empty_cache()
    assert worst > 1e-13
