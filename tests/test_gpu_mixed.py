"""Mixed precision (FP32 far pairs, FP64 near and singular pairs) against the FP64
oracle: relative Frobenius error <= 1e-6, the accuracy bar of the mixed mode."""

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import Precision
from ndgrid.grid import Grid

from test_gpu_parity import gpu_assemble, oracle_assemble, rel_err

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


@pytest.mark.parametrize("kernel,op,k", [
    ("laplace", "single_layer", 0.0),
    ("laplace", "double_layer", 0.0),
    ("laplace", "adjoint_double_layer", 0.0),
    ("helmholtz", "single_layer", 8.0),
    ("helmholtz", "double_layer", 8.0),
    ("helmholtz", "adjoint_double_layer", 8.0),
    ("helmholtz", "single_layer", 20.0),   # |k delta| > 0.8 somewhere: sincosf branch
    # k (max rad_x + max rad_y) = 0.39 and 0.78: small-phase launches (no reduction)
    ("helmholtz", "single_layer", 2.0),
    ("helmholtz", "single_layer", 4.0),
    ("helmholtz", "double_layer", 4.0),
])
def test_mixed_dp0_matches_oracle(kernel, op, k):
    pts, cells = shapes.icosphere(3)
    pts = shapes.radial_perturbation(pts, seed=3)
    grid = Grid(pts, cells)
    a = gpu_assemble(grid, kernel, op, k, precision=Precision.Mixed)
    o = oracle_assemble(grid, kernel, op, k)
    err = rel_err(a, o)
    assert err <= MIXED_TOL
    # the FP32 path really ran (an all-FP64 result would agree to ~1e-15)
    assert err > 1e-13


def test_mixed_far_from_origin():
    """Centroid-relative FP32 coordinates keep the accuracy for a mesh far from the
    origin (absolute FP32 coordinates would lose ~1e-4 here)."""
    pts, cells = shapes.icosphere(3)
    grid = Grid(pts + np.array([1.0e3, -2.0e3, 5.0e2]), cells)
    a = gpu_assemble(grid, "laplace", "single_layer", precision=Precision.Mixed)
    o = oracle_assemble(grid, "laplace", "single_layer")
    assert rel_err(a, o) <= MIXED_TOL


@pytest.mark.parametrize("kernel,op,k", [
    ("laplace", "double_layer", 0.0),
    ("laplace", "adjoint_double_layer", 0.0),
    ("laplace", "hypersingular", 0.0),
    ("helmholtz", "double_layer", 8.0),
    ("helmholtz", "hypersingular", 8.0),
    ("helmholtz", "adjoint_double_layer", 4.0),
    ("helmholtz", "hypersingular", 2.0),
])
def test_mixed_p1_matches_oracle(kernel, op, k):
    pts, cells = shapes.icosphere(3)
    pts = shapes.radial_perturbation(pts, seed=4)
    grid = Grid(pts, cells)
    sp = (1, True)
    a = gpu_assemble(grid, kernel, op, k, test=sp, trial=sp, precision=Precision.Mixed)
    o = oracle_assemble(grid, kernel, op, k, test=sp, trial=sp)
    err = rel_err(a, o)
    assert 1e-13 < err <= MIXED_TOL


@pytest.mark.parametrize("kernel,op,k,sp", [
    ("helmholtz", "single_layer", 8.0, (0, False)),
    ("laplace", "hypersingular", 0.0, (1, True)),
    ("laplace", "double_layer", 0.0, (1, True)),
    ("laplace", "adjoint_double_layer", 0.0, (1, True)),
    ("laplace", "double_layer", 0.0, (1, False)),
    ("helmholtz", "double_layer", 5.0, (1, True)),
    ("helmholtz", "adjoint_double_layer", 5.0, (1, True)),
    ("helmholtz", "double_layer", 8.0, (1, True)),
])
def test_mixed_one_space_symmetric(kernel, op, k, sp):
    """The mixed path on one space object: lower-triangle (mirrored) tile pairs for the
    single layer and the hypersingular operator; for the double layer and its adjoint on
    P1 / DP1 the tile pairs tx >= sy, each far pair in both orders from one FP32 kernel
    value (Helmholtz when every phase stays in the polynomial range: k = 5 here; k = 8
    exceeds it on this mesh and takes the one-order launch)."""
    pts, cells = shapes.icosphere(3)
    grid = Grid(shapes.radial_perturbation(pts, seed=12), cells)
    a = gpu_assemble(grid, kernel, op, k, test=sp, trial=sp, precision=Precision.Mixed,
                     one_space=True)
    o = oracle_assemble(grid, kernel, op, k, test=sp, trial=sp)
    err = rel_err(a, o)
    assert 1e-13 < err <= MIXED_TOL

