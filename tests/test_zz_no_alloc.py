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


def _meshes():
    pts, cells = shapes.icosphere(3)
    test = (shapes.radial_perturbation(pts, seed=11), cells)
    trial = (shapes.radial_perturbation(pts, seed=12) + np.array([2.5, 0.3, -0.4]), cells)
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


def _noalloc(test, trial, kernel, op, k, q):
    import torch

    tp = torch.tensor(test[0], dtype=torch.float64, device="cuda")
    tc = torch.tensor(test[1], dtype=torch.int32, device="cuda")
    sp = torch.tensor(trial[0], dtype=torch.float64, device="cuda")
    sc = torch.tensor(trial[1], dtype=torch.int32, device="cuda")
    dt = torch.float64 if kernel == 0 else torch.complex128
    out = torch.full((len(trial[1]), len(test[1])), float("nan"), dtype=dt, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.bempp_assemble_regular_dp0_noalloc(
        kernel, op.value, k, lib.Precision_FP64, q,
        ffi.cast("double*", tp.data_ptr()), len(test[0]), ffi.cast("int32_t*", tc.data_ptr()),
        len(test[1]), ffi.cast("double*", sp.data_ptr()), len(trial[0]),
        ffi.cast("int32_t*", sc.data_ptr()), len(trial[1]), ffi.cast("void*", out.data_ptr()),
        ffi.cast("void*", stream))
    assert st == lib.BemppStatus_Ok, _lib.last_error()
    torch.cuda.synchronize()
    return out.T.cpu().numpy()


def test_no_alloc_matches_existing_entry_point_twice():
    import torch

    torch.cuda.set_device(0)
    test, trial = _meshes()
    cases = [(0, OperatorType.SingleLayer, 0.0, 6), (1, OperatorType.DoubleLayer, 5.0, 6)]
    for kernel, op, k, q in cases:  # two calls in a row share the scratch array
        ref = _existing(test, trial, kernel, op, k, q)
        got = _noalloc(test, trial, kernel, op, k, q)
        assert np.all(np.isfinite(got))
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= TOL, (kernel, op, err)


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
