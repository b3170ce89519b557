"""The allocation-free entry point bempp_assemble_regular_dp0_noalloc.

It serves callers that cannot let a library allocate GPU memory (fixed memory budgets,
custom pools, no allocation after start-up): they pass device buffers for the inputs and
the output, and the library's scratch lives in a static device array.  Its result must
equal what the ordinary entry point computes for the same problem: spaces on two
different grid objects, assembled with boundary_assembler_assemble_into_device.  Two
calls in a row are checked, because every call reuses the same scratch array.

This file is named so that pytest collects it last.
"""

import numpy as np
import pytest

from bempp import _lib, shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,
                                     create_helmholtz_assembler, create_laplace_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

pytestmark = pytest.mark.gpu

TOL = 1e-12
ffi, lib = _lib.ffi, _lib.lib


MIXED_TOL = 1e-6  # the mixed-precision tolerance of tests/test_gpu_mixed.py


def _meshes(offset=(2.5, 0.3, -0.4), level=3):
    pts, cells = shapes.icosphere(level)
    test = (shapes.radial_perturbation(pts, seed=11), cells)
    trial = (shapes.radial_perturbation(pts, seed=12) + np.array(offset), cells)
    return test, trial


def _existing(test, trial, kernel, op, k, q):
    import torch

    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, q)
    fam = create_family(Family.Lagrange, 0, Continuity.Discontinuous)
    ts = function_space(Grid(*test), fam)
    ss = function_space(Grid(*trial), fam)
    a = (create_laplace_assembler(op, opts) if kernel == 0
         else create_helmholtz_assembler(op, k, opts))
    dt = torch.float64 if kernel == 0 else torch.complex128
    out = torch.zeros((ss.global_size, ts.global_size), dtype=dt, device="cuda")
    a.assemble_into_device(ss, ts, out, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.T.cpu().numpy()  # (n_test, n_trial)


def _call(test, trial, kernel, op, k, q, precision, out):
    import torch

    tp = torch.tensor(np.asarray(test[0]), dtype=torch.float64, device="cuda")
    tc = torch.tensor(np.asarray(test[1]), dtype=torch.int32, device="cuda")
    sp = torch.tensor(np.asarray(trial[0]), dtype=torch.float64, device="cuda")
    sc = torch.tensor(np.asarray(trial[1]), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    return lib.bempp_assemble_regular_dp0_noalloc(
        kernel, op.value, k, precision, q,
        ffi.cast("double*", tp.data_ptr()), len(test[0]), ffi.cast("int32_t*", tc.data_ptr()),
        len(test[1]), ffi.cast("double*", sp.data_ptr()), len(trial[0]),
        ffi.cast("int32_t*", sc.data_ptr()), len(trial[1]), ffi.cast("void*", out.data_ptr()),
        ffi.cast("void*", stream))


def _noalloc(test, trial, kernel, op, k, q, precision=None):
    import torch

    if precision is None:
        precision = lib.Precision_FP64
    dt = torch.float64 if kernel == 0 else torch.complex128
    out = torch.full((len(trial[1]), len(test[1])), float("nan"), dtype=dt, device="cuda")
    st = _call(test, trial, kernel, op, k, q, precision, out)
    assert st == lib.BemppStatus_Ok, _lib.last_error()
    torch.cuda.synchronize()
    return out.T.cpu().numpy()


def _rel(got, ref):
    return np.linalg.norm(got - ref) / np.linalg.norm(ref)


def test_no_alloc_matches_existing_entry_point_twice():
    import torch

    torch.cuda.set_device(0)
    test, trial = _meshes()
    cases = [(0, OperatorType.SingleLayer, 0.0, 6), (1, OperatorType.DoubleLayer, 5.0, 6)]
    for kernel, op, k, q in cases:  # two calls in a row share the scratch array
        ref = _existing(test, trial, kernel, op, k, q)
        got = _noalloc(test, trial, kernel, op, k, q)
        assert np.all(np.isfinite(got))
        err = _rel(got, ref)
        assert err <= TOL, (kernel, op, err)


# (kernel, operator, k, regular points, mixed precision, trial offset)
CASES = [
    (0, OperatorType.AdjointDoubleLayer, 0.0, 6, False, (2.5, 0.3, -0.4)),
    (1, OperatorType.SingleLayer, 4.0, 7, False, (2.5, 0.3, -0.4)),   # odd rule
    (1, OperatorType.AdjointDoubleLayer, 8.0, 3, False, (2.1, 0.0, 0.0)),
    # mixed precision: FP32 far pairs, near pairs (the meshes are 0.06 apart) queued in
    # the kernel and integrated in FP64, every Helmholtz phase reduced
    (0, OperatorType.SingleLayer, 0.0, 6, True, (2.1, 0.0, 0.0)),
    (0, OperatorType.DoubleLayer, 0.0, 7, True, (2.1, 0.0, 0.0)),
    (1, OperatorType.SingleLayer, 5.0, 6, True, (2.1, 0.0, 0.0)),
    (1, OperatorType.AdjointDoubleLayer, 8.0, 6, True, (2.5, 0.3, -0.4)),
    (1, OperatorType.DoubleLayer, 12.0, 7, True, (2.1, 0.0, 0.0)),
]


@pytest.mark.parametrize("kernel,op,k,q,mixed,offset", CASES)
def test_no_alloc_operators_rules_and_precisions(kernel, op, k, q, mixed, offset):
    test, trial = _meshes(offset)
    ref = _existing(test, trial, kernel, op, k, q)
    prec = lib.Precision_Mixed if mixed else lib.Precision_FP64
    for _ in range(2):
        got = _noalloc(test, trial, kernel, op, k, q, prec)
        err = _rel(got, ref)
        if mixed:
            assert 1e-13 < err <= MIXED_TOL, (kernel, op, k, q, err)
        else:
            assert err <= TOL, (kernel, op, k, q, err)


def test_no_alloc_cell_counts_off_the_tile_size():
    """1,000 test and 777 trial cells: neither a multiple of the 32-cell tile."""
    test, trial = _meshes()
    test = (test[0], test[1][:1000])
    trial = (trial[0], trial[1][:777])
    for kernel, op, k in ((0, OperatorType.DoubleLayer, 0.0), (1, OperatorType.SingleLayer, 3.0)):
        ref = _existing(test, trial, kernel, op, k, 6)
        got = _noalloc(test, trial, kernel, op, k, 6)
        assert got.shape == (1000, 777)
        assert _rel(got, ref) <= TOL


def test_no_alloc_at_its_cell_limit():
    """8,192 cells per mesh (the refined octahedron of level 5) is the largest size."""
    pts, cells = shapes.regular_sphere(5)
    assert len(cells) == 8192
    test = (pts, cells)
    trial = (pts * 0.5 + np.array([3.0, 0.0, 0.0]), cells)
    ref = _existing(test, trial, 0, OperatorType.SingleLayer, 0.0, 3)
    got = _noalloc(test, trial, 0, OperatorType.SingleLayer, 0.0, 3)
    assert _rel(got, ref) <= TOL


def test_no_alloc_rejects_out_of_range_vertex_indices():
    """An index outside [0, npoints) is found by the device check before any point is
    read: the call fails with InvalidArgument and leaves the output untouched; the next
    valid call works."""
    import torch

    test, trial = _meshes()
    bad_cells = np.array(trial[1])
    bad_cells[17, 1] = len(trial[0])      # one past the end
    bad_cells[300, 2] = -4                # negative
    out = torch.full((len(trial[1]), len(test[1])), 7.0, dtype=torch.float64, device="cuda")
    st = _call(test, (trial[0], bad_cells), 0, OperatorType.SingleLayer, 0.0, 6,
               lib.Precision_FP64, out)
    assert st == lib.BemppStatus_InvalidArgument
    assert "2 cell vertex index" in _lib.last_error()
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
    ref = _existing(test, trial, 0, OperatorType.SingleLayer, 0.0, 6)
    assert _rel(_noalloc(test, trial, 0, OperatorType.SingleLayer, 0.0, 6), ref) <= TOL


def test_no_alloc_rejects_sizes_beyond_its_limit():
    import torch

    torch.cuda.set_device(0)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ffi.cast("void*", dummy.data_ptr())
    st = lib.bempp_assemble_regular_dp0_noalloc(
        0, lib.OperatorType_SingleLayer, 0.0, lib.Precision_FP64, 6, ffi.cast("double*", p), 3,
        ffi.cast("int32_t*", p), 8193, ffi.cast("double*", p), 3, ffi.cast("int32_t*", p), 1,
        p, ffi.NULL)
    assert st == lib.BemppStatus_InvalidArgument
    assert "8192" in _lib.last_error()
    st = lib.bempp_assemble_regular_dp0_noalloc(
        0, lib.OperatorType_SingleLayer, 0.0, lib.Precision_FP64, 37, ffi.cast("double*", p), 3,
        ffi.cast("int32_t*", p), 1, ffi.cast("double*", p), 3, ffi.cast("int32_t*", p), 1,
        p, ffi.NULL)
    assert st == lib.BemppStatus_InvalidArgument
