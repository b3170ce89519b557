"""Host-memory assembly (BoundaryAssembler.assemble -> boundary_assembler_assemble_into_memory_ex)
on matrices large enough to be assembled in several chunks of trial tiles, with the
device-to-host copy of finished columns overlapped: the result must equal the
single-launch device assembly (assemble_into_device) of the same operator.  Every case
runs twice: into a page-locked output (direct DMA of finished columns) and into a
pageable numpy array (pinned staging ring and host copy threads).

DP0 x DP0 entries are written by one kernel and one singular add each, so the chunked
result is bit-identical; P1 entries are sums of atomic adds whose order differs between
launches, so they agree to rounding (relative Frobenius <= 1e-13).  A row subset of the
largest case is also checked against the FP64 oracle.
"""

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,
                                     create_helmholtz_assembler, create_laplace_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

from test_gpu_parity import oracle_assemble, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["page_locked", "pageable"], autouse=True)
def output_memory(request, monkeypatch):
    from bempp.assembly import boundary

    if request.param == "pageable":
        monkeypatch.setattr(boundary, "PINNED_OUTPUT_MIN_BYTES", None)
    return request.param

OPS = {"single_layer": OperatorType.SingleLayer, "double_layer": OperatorType.DoubleLayer,
       "adjoint_double_layer": OperatorType.AdjointDoubleLayer,
       "hypersingular": OperatorType.Hypersingular}


def boundary_pinned():
    from bempp.assembly import boundary

    return boundary.PINNED_OUTPUT_MIN_BYTES is not None


def assemble_both(level, kernel, op, k, degree, dtype, precision=None):
    import torch

    pts, cells = shapes.icosphere(level)
    grid = Grid(shapes.radial_perturbation(pts, seed=level), cells)
    real = np.float32 if dtype in (np.float32, np.complex64) else np.float64
    fam = create_family(Family.Lagrange, degree,
                        Continuity.Standard if degree else Continuity.Discontinuous, real)
    sp = function_space(grid, fam)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    if precision is not None:
        opts.set_precision(precision)
    if kernel == "laplace":
        a = create_laplace_assembler(OPS[op], opts, dtype)
    else:
        a = create_helmholtz_assembler(OPS[op], k, opts, dtype)
    host = a.assemble(sp, sp)
    if boundary_pinned():
        assert type(host.base).__name__ == "_PageLockedBlock"
    n = sp.global_size
    tdt = {np.float64: torch.float64, np.float32: torch.float32,
           np.complex128: torch.complex128, np.complex64: torch.complex64}[dtype]
    dev = torch.empty((n, n), dtype=tdt, device="cuda")  # row-major view of the column-major A
    a.assemble_into_device(sp, sp, dev, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return grid, host, dev.cpu().numpy().T


@pytest.mark.parametrize("level,kernel,op,k,dtype", [
    (4, "helmholtz", "single_layer", 8.0, np.complex128),   # 419 MB: 5 chunks
    (4, "laplace", "double_layer", 0.0, np.float32),        # 105 MB: 2 chunks, converted per chunk
])
def test_chunked_dp0_is_bit_identical(level, kernel, op, k, dtype):
    _, host, dev = assemble_both(level, kernel, op, k, 0, dtype)
    assert host.dtype == dtype
    assert np.array_equal(host, dev)


def test_chunked_p1_matches_device_and_oracle():
    # 10242^2 doubles = 839 MB: 9 chunks whose finished columns are scattered runs
    grid, host, dev = assemble_both(5, "laplace", "double_layer", 0.0, 1, np.float64)
    assert rel_err(host, dev) <= 1e-13
    from oracle import oracle

    rows = np.random.default_rng(9).choice(host.shape[0], size=24, replace=False)
    # the oracle's regular part restricted to the cells holding those DOFs: their rows
    # are complete
    dofs, _ = oracle.cell_dofs(grid.points, grid.cells, 1, True)
    cells = np.flatnonzero(np.isin(dofs, rows).any(axis=1))
    o = oracle_assemble(grid, "laplace", "double_layer", test=(1, True), trial=(1, True),
                        test_subset=cells)
    assert rel_err(host[rows], o[rows]) <= 1e-12


@pytest.mark.parametrize("op", ["hypersingular", "double_layer", "adjoint_double_layer"])
def test_chunked_p1_helmholtz(op):
    # 2562^2 complex128 = 105 MB: 3 chunks (hypersingular: of tile pairs tx >= sy)
    _, host, dev = assemble_both(4, "helmholtz", op, 5.0, 1, np.complex128)
    assert rel_err(host, dev) <= 1e-13


@pytest.mark.parametrize("kernel,k", [("laplace", 0.0), ("helmholtz", 5.0)])
def test_chunked_p1_mixed_double_layer(kernel, k):
    from bempp.assembly.boundary import Precision

    # the chunked call runs the full tile grid, the device call the paired launch: two
    # FP32 formulations, each within ~2e-8 of the FP64 matrix, so they agree to the mixed
    # tolerance, not to rounding
    dtype = np.float64 if kernel == "laplace" else np.complex128
    _, host, dev = assemble_both(4, kernel, "double_layer", k, 1, dtype, Precision.Mixed)
    assert rel_err(host, dev) <= 1e-6


def test_chunked_p1_laplace_adjoint_double_layer():
    _, host, dev = assemble_both(5, "laplace", "adjoint_double_layer", 0.0, 1, np.float64)
    assert rel_err(host, dev) <= 1e-13


def test_page_locked_result_outlives_the_next_assembly():
    """A kept result is not reused for the next one (its block stays alive)."""
    _, first, _ = assemble_both(4, "laplace", "double_layer", 0.0, 0, np.float64)
    keep = first.copy()
    _, second, _ = assemble_both(4, "laplace", "single_layer", 0.0, 0, np.float64)
    assert np.array_equal(first, keep)
    assert not np.array_equal(first, second)



def test_device_blocks_of_freed_grids_are_reused_and_trimmed(output_memory):
    """Device blocks of a freed grid, space and assembler go to the library's cache: the
    next ones reuse them (same result), and bempp_device_trim hands them back."""
    import gc

    import torch

    from bempp._lib import lib

    if output_memory != "page_locked":
        pytest.skip("one memory kind is enough")

    def once():
        pts, cells = shapes.icosphere(3)
        grid = Grid(shapes.radial_perturbation(pts, seed=3), cells)
        sp = function_space(grid, create_family(Family.Lagrange, 0, Continuity.Discontinuous))
        opts = BoundaryAssemblerOptions()
        opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
        a = create_laplace_assembler(OPS["single_layer"], opts, np.float64)
        n = sp.global_size
        dev = torch.empty((n, n), dtype=torch.float64, device="cuda")
        a.assemble_into_device(sp, sp, dev, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return dev.cpu().numpy()

    lib.bempp_device_trim()
    first = once()
    gc.collect()
    second = once()
    assert np.array_equal(first, second)
    gc.collect()
    assert lib.bempp_device_trim() > 0
    assert lib.bempp_device_trim() == 0
