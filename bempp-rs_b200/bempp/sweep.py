"""Batched Helmholtz single-layer frequency sweep (one persistent, graph-captured launch).

``helmholtz_single_layer_sweep(grids, wavenumbers)`` assembles the DP0 x DP0 Helmholtz
single-layer matrix of every grid at every wavenumber: far pairs in FP32, near and
singular pairs in FP64, complex64 results.  It returns one CUDA tensor per grid of shape
(nk, n, n) holding the transposed matrices (column-major storage), so ``out[i][j].T`` is
the matrix of grid i at wavenumber j.
"""

from __future__ import annotations

import numpy as np

from bempp._lib import check as _check
from bempp._lib import ffi as _ffi
from bempp._lib import lib as _lib
from bempp.assembly.boundary import BoundaryAssemblerOptions
from bempp.function_space import grid_handle
from ndelement.reference_cell import ReferenceCellType


def helmholtz_single_layer_sweep(grids, wavenumbers, outputs=None, stream=None,
                                 singular_order: int = 4):
    import torch

    ks = np.ascontiguousarray(wavenumbers, dtype=np.float64)
    owners = [grid_handle(g) for g in grids]  # held until the call returns
    handles = [o.ptr for o in owners]
    if outputs is None:
        outputs = [torch.empty((len(ks), len(g.cells), len(g.cells)), dtype=torch.complex64,
                               device="cuda") for g in grids]
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    opts.set_singular_quadrature_degree(ReferenceCellType.Triangle, ReferenceCellType.Triangle,
                                        singular_order)
    gh = _ffi.new("GridT*[]", handles)
    oh = _ffi.new("void*[]", [_ffi.cast("void*", o.data_ptr()) for o in outputs])
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    _check(_lib.bempp_helmholtz_single_layer_dp0_sweep_device(
        gh, len(handles), _ffi.cast("double*", ks.ctypes.data), len(ks), opts._rs_options, oh,
        _ffi.cast("void*", int(stream))), "sweep")
    return outputs


def set_tuning(kchunk: int = 0, blocks_per_sm: int = 4, tile_shape: int = 1):
    """Fix the sweep's launch parameters (kchunk = 0: autotune again)."""
    _check(_lib.bempp_sweep_set_tuning(kchunk, blocks_per_sm, tile_shape), "sweep tuning")


def last_tuning():
    """(wavenumbers per work item, CTAs per SM, probe ms per (tile pair, wavenumber),
    tile shape) of the last sweep."""
    k = _ffi.new("int32_t*")
    b = _ffi.new("int32_t*")
    s = _ffi.new("int32_t*")
    t = _ffi.new("double*")
    _check(_lib.bempp_sweep_last_tuning(k, b, s, t), "sweep tuning")
    return int(k[0]), int(b[0]), float(t[0]), int(s[0])
