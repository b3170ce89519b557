"""Differentiable Helmholtz single-layer energy (adjoint gradient on the GPU).

J(x, k) = Re(lambda^H A(x, k) mu) for the Helmholtz single-layer operator on DP0 x DP0
spaces of a flat-triangle mesh with vertex coordinates x.  The gradient with respect to
every coordinate and to k comes from one adjoint pass of the library
(``bempp_helmholtz_single_layer_dp0_gradient_device``), which differentiates the
discrete quadrature sums directly and never forms dA/dx.

    energy = HelmholtzSingleLayerEnergy.apply(points, k, lam, mu, cells)
    energy.backward()          # points.grad, k.grad

points: (npoints, 3) float64 tensor (CPU or CUDA, requires_grad as needed); k: 0-d
float64 tensor; lam, mu: (ncells,) complex128 tensors (constants); cells: (ncells, 3)
integer array of point indices.
"""

from __future__ import annotations

import numpy as np
import torch

from bempp._lib import check as _check
from bempp._lib import ffi as _ffi
from bempp._lib import lib as _lib
from bempp.assembly.boundary import BoundaryAssemblerOptions, check_device
from ndelement.reference_cell import ReferenceCellType


def _grid(points: np.ndarray, cells: np.ndarray):
    pts = np.ascontiguousarray(points, dtype=np.float64)
    cls = np.ascontiguousarray(cells, dtype=np.uintp)
    g = _lib.bempp_grid_from_points_cells(_ffi.cast("void*", pts.ctypes.data), len(pts),
                                          _lib.DType_F64, _ffi.cast("size_t*", cls.ctypes.data),
                                          len(cls))
    if g == _ffi.NULL:
        raise ValueError(_ffi.string(_lib.bempp_last_error()).decode())
    return g


def energy_and_gradient(points, cells, k, lam, mu, regular_points=6, singular_order=4,
                        device=None, mixed=False):
    """J, dJ/dk and dJ/dpoints (npoints x 3) as torch float64 tensors on `device`; with
    mixed=True far pairs are integrated in FP32 (near and singular pairs stay FP64)."""
    from bempp.assembly.boundary import Precision

    device = torch.device("cuda") if device is None else torch.device(device)
    pts = points.detach().cpu().numpy() if torch.is_tensor(points) else np.asarray(points)
    cls = cells.cpu().numpy() if torch.is_tensor(cells) else np.asarray(cells)
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, regular_points)
    opts.set_singular_quadrature_degree(ReferenceCellType.Triangle, ReferenceCellType.Triangle,
                                        singular_order)
    opts.set_precision(Precision.Mixed if mixed else Precision.FP64)
    g = _grid(pts, cls)
    try:
        lam_d = torch.as_tensor(lam, dtype=torch.complex128, device=device).contiguous()
        mu_d = torch.as_tensor(mu, dtype=torch.complex128, device=device).contiguous()
        out = torch.zeros(2, dtype=torch.float64, device=device)
        grad = torch.zeros((len(pts), 3), dtype=torch.float64, device=device)
        stream = torch.cuda.current_stream(device).cuda_stream
        _check(_lib.bempp_helmholtz_single_layer_dp0_gradient_device(
            g, opts._rs_options, float(k), _ffi.cast("void*", lam_d.data_ptr()),
            _ffi.cast("void*", mu_d.data_ptr()), _ffi.cast("double*", out.data_ptr()),
            _ffi.cast("double*", grad.data_ptr()), _ffi.cast("void*", stream)),
            "adjoint gradient")
        # waits for the stream; raises if a block's tile copies timed out (its pairs
        # would be missing from the gradient)
        check_device(stream)
    finally:
        _lib.grid_t_free_bempp(g)
    return out[0], out[1], grad


class HelmholtzSingleLayerEnergy(torch.autograd.Function):
    """J = Re(lambda^H A(points, k) mu) with a hand-written adjoint backward."""

    @staticmethod
    def forward(ctx, points, k, lam, mu, cells):
        value, dk, grad = energy_and_gradient(points, cells, float(k), lam, mu)
        ctx.save_for_backward(grad.to(points.device), dk.to(k.device))
        return value.to(points.device)

    @staticmethod
    def backward(ctx, g):
        grad, dk = ctx.saved_tensors
        return g * grad, g * dk, None, None, None
