"""Failure reporting of the regular kernels' bounded wait, on the GPU without a fault.

Each block of the regular kernels waits (boundedly) for the bulk copies that stage its
two cell tiles in shared memory.  A test hook lowers the number of polls of that first
wait to zero, so every block gives up at once: it records the failure in a device
counter, drains its copies with a second full-length wait and returns without writing.
The device entry point must then report BemppStatus_Incomplete through
bempp_device_status (and leave the output untouched), the host entry point must raise,
and once the limit is back the next assembly must match the FP64 oracle.  The adjoint
gradient's regular kernel stages its tiles the same way and reports the same way.
"""

import numpy as np
import pytest

from bempp import _lib, shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType, check_device,
                                     create_laplace_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

from test_gpu_parity import oracle_two_grids, rel_err

pytestmark = pytest.mark.gpu

ffi, lib = _lib.ffi, _lib.lib
DEFAULT_POLLS = 1 << 22


@pytest.fixture
def stage_polls():
    def set_polls(n):
        assert lib.bempp_set_stage_wait_limit(n) == lib.BemppStatus_Ok, _lib.last_error()

    try:
        yield set_polls
    finally:
        set_polls(DEFAULT_POLLS)
        lib.bempp_device_status(ffi.NULL)  # drop any count left behind


def _spaces_on_two_grids():
    """DP0 spaces on two grid objects: every entry comes from the regular kernel."""
    pts, cells = shapes.icosphere(3)
    g1 = Grid(shapes.radial_perturbation(pts, seed=3), cells)
    g2 = Grid(shapes.radial_perturbation(pts, seed=4) + np.array([3.0, 0.0, 0.0]), cells)
    fam = create_family(Family.Lagrange, 0, Continuity.Discontinuous)
    return g1, g2, function_space(g1, fam), function_space(g2, fam)


def test_device_path_reports_a_wait_that_ran_out(stage_polls):
    import torch

    g1, g2, test, trial = _spaces_on_two_grids()
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    a = create_laplace_assembler(OperatorType.SingleLayer, opts)
    n = len(g1.cells)
    out = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.bempp_device_status(ffi.cast("void*", stream)) == lib.BemppStatus_Ok

    stage_polls(0)
    a.assemble_into_device(trial, test, out, stream)
    st = lib.bempp_device_status(ffi.cast("void*", stream))
    assert st == lib.BemppStatus_Incomplete
    assert "tile blocks timed out" in _lib.last_error()
    assert bool(torch.isnan(out).all()), "a block that gave up wrote entries"
    # the count was reset by the check
    assert lib.bempp_device_status(ffi.cast("void*", stream)) == lib.BemppStatus_Ok

    stage_polls(DEFAULT_POLLS)
    a.assemble_into_device(trial, test, out, stream, check=True)
    m = out.T.cpu().numpy()
    # the same regular part from the oracle: test cells of g1 against trial cells of g2
    o = oracle_two_grids(g1, g2, "laplace", "single_layer")
    assert rel_err(m, o) <= 1e-12


def test_host_path_raises_on_a_wait_that_ran_out(stage_polls):
    g1, g2, test, trial = _spaces_on_two_grids()
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    a = create_laplace_assembler(OperatorType.SingleLayer, opts)
    stage_polls(0)
    with pytest.raises(RuntimeError, match="status 7"):
        a.assemble(trial, test)
    stage_polls(DEFAULT_POLLS)
    assert rel_err(a.assemble(trial, test), oracle_two_grids(g1, g2, "laplace", "single_layer")) <= 1e-12


def test_check_device_raises_after_a_wait_that_ran_out(stage_polls):
    import torch

    g1, g2, test, trial = _spaces_on_two_grids()
    a = create_laplace_assembler(OperatorType.DoubleLayer)
    n = len(g1.cells)
    out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    stage_polls(0)
    with pytest.raises(RuntimeError, match="timed out"):
        a.assemble_into_device(trial, test, out, None, check=True)
    check_device(None)  # the count was taken by the failed check


def test_adjoint_gradient_reports_a_wait_that_ran_out(stage_polls):
    import torch

    from bempp.autograd import energy_and_gradient

    pts, cells = shapes.icosphere(2)
    pts = shapes.radial_perturbation(pts, seed=8)
    rng = np.random.default_rng(1)
    lam = rng.standard_normal(len(cells)) + 1j * rng.standard_normal(len(cells))
    mu = rng.standard_normal(len(cells)) + 1j * rng.standard_normal(len(cells))
    j0, dk0, g0 = energy_and_gradient(pts, cells, 2.0, lam, mu)
    stage_polls(0)
    with pytest.raises(RuntimeError, match="timed out"):
        energy_and_gradient(pts, cells, 2.0, lam, mu)
    stage_polls(DEFAULT_POLLS)
    j1, dk1, g1 = energy_and_gradient(pts, cells, 2.0, lam, mu)
    assert float(j1) == float(j0) or abs(float(j1) - float(j0)) <= 1e-12 * abs(float(j0))
    assert torch.allclose(g1, g0, rtol=1e-12, atol=1e-12 * float(g0.abs().max()))
