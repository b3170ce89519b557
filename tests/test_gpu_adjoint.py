"""Adjoint gradient of J = Re(lambda^H A(x, k) mu), Helmholtz single layer, DP0, k = 5, on
the 5,120-triangle icosphere with a seeded radial perturbation (seed 5120), lambda and mu
complex standard normal (seed 5, lambda first).

Checks: J equals Re(lambda^H A mu) with A from the dense FP64 assembly; the gradient
matches central finite differences (h = 1e-6) of that FP64 forward on 64 coordinates drawn
with seed 64, and in k; the torch.autograd.Function returns the same gradient.
"""

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,
                                     create_helmholtz_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

pytestmark = pytest.mark.gpu

K = 5.0


def problem(level=4):
    pts, cells = shapes.icosphere(level)
    pts = shapes.radial_perturbation(pts, seed=5120)
    rng = np.random.default_rng(5)
    n = len(cells)
    lam = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    mu = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return pts, cells, lam, mu


def forward_j(pts, cells, k, lam, mu):
    """Re(lambda^H A mu) from the dense FP64 assembly on the device."""
    import torch

    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    a = create_helmholtz_assembler(OperatorType.SingleLayer, k, opts)
    sp = function_space(Grid(pts, cells), create_family(Family.Lagrange, 0, Continuity.Discontinuous))
    n = sp.global_size
    out = torch.empty((n, n), dtype=torch.complex128, device="cuda")  # column-major A as A^T
    a.assemble_into_device(sp, sp, out, torch.cuda.current_stream().cuda_stream)
    lam_t = torch.as_tensor(lam, device="cuda")
    mu_t = torch.as_tensor(mu, device="cuda")
    # out holds A^T (row j = column j of A): A mu = out^T mu
    amu = out.T @ mu_t
    return float(torch.real(torch.vdot(lam_t, amu)).item())


def test_value_matches_dense_forward():
    from bempp.autograd import energy_and_gradient

    pts, cells, lam, mu = problem(3)
    j, _, _ = energy_and_gradient(pts, cells, K, lam, mu)
    ref = forward_j(pts, cells, K, lam, mu)
    assert abs(j.item() - ref) <= 1e-12 * abs(ref)


def test_gradient_matches_central_differences():
    from bempp.autograd import energy_and_gradient

    pts, cells, lam, mu = problem(4)
    _, dk, grad = energy_and_gradient(pts, cells, K, lam, mu)
    grad = grad.cpu().numpy().ravel()
    idx = np.random.default_rng(64).choice(pts.size, size=64, replace=False)
    h = 1e-6
    fd = []
    for c in idx:
        p1 = pts.copy().ravel()
        p2 = pts.copy().ravel()
        p1[c] += h
        p2[c] -= h
        fd.append((forward_j(p1.reshape(-1, 3), cells, K, lam, mu) -
                   forward_j(p2.reshape(-1, 3), cells, K, lam, mu)) / (2 * h))
    fd = np.array(fd)
    scale = np.abs(grad).max()
    err = np.abs(fd - grad[idx]).max() / scale
    assert err <= 1e-6, err
    fdk = (forward_j(pts, cells, K + h, lam, mu) - forward_j(pts, cells, K - h, lam, mu)) / (2 * h)
    assert abs(fdk - dk.item()) <= 1e-6 * max(abs(fdk), 1.0)


def test_autograd_function():
    import torch

    from bempp.autograd import HelmholtzSingleLayerEnergy, energy_and_gradient

    pts, cells, lam, mu = problem(3)
    x = torch.tensor(pts, dtype=torch.float64, requires_grad=True)
    k = torch.tensor(K, dtype=torch.float64, requires_grad=True)
    j = HelmholtzSingleLayerEnergy.apply(x, k, torch.as_tensor(lam), torch.as_tensor(mu), cells)
    (2.0 * j).backward()
    jv, dk, grad = energy_and_gradient(pts, cells, K, lam, mu)
    # two adjoint passes agree up to the order of their atomic additions
    assert abs(j.item() - jv.item()) <= 1e-12 * abs(jv.item())
    g = grad.cpu().numpy()
    assert np.abs(x.grad.numpy() - 2.0 * g).max() <= 1e-12 * np.abs(g).max()
    assert abs(k.grad.item() - 2.0 * dk.item()) <= 1e-12 * abs(dk.item())


def test_mixed_gradient_matches_fp64_gradient():
    """Mixed precision (FP32 far pairs): J and the gradient agree with the FP64 adjoint."""
    from bempp.autograd import energy_and_gradient

    pts, cells, lam, mu = problem(4)
    j64, dk64, g64 = energy_and_gradient(pts, cells, K, lam, mu)
    jm, dkm, gm = energy_and_gradient(pts, cells, K, lam, mu, mixed=True)
    g64 = g64.cpu().numpy()
    gm = gm.cpu().numpy()
    assert abs(jm.item() - j64.item()) <= 1e-6 * abs(j64.item())
    err = np.abs(gm - g64).max() / np.abs(g64).max()
    assert 1e-13 < err <= 1e-5, err
    assert abs(dkm.item() - dk64.item()) <= 1e-5 * abs(dk64.item())
