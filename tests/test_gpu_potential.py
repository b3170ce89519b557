"""Off-surface potential operators on the GPU (potential.cu through the C-ABI) against
the CPU oracle (oracle/potential.py) and against the bempp-cl values of the reference's
commented potential tests (tests/compare_to_bempp_cl.rs:208-320)."""

import json
import os

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import BoundaryAssemblerOptions, OperatorType
from bempp.assembly.potential import (create_helmholtz_potential_assembler,
                                      create_laplace_potential_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

pytestmark = pytest.mark.gpu

OPS = {"single_layer": OperatorType.SingleLayer, "double_layer": OperatorType.DoubleLayer}
FP64_TOL = 1e-12


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def assembler(kernel, op, k, q=None, dtype=None):
    opts = BoundaryAssemblerOptions()
    if q is not None:
        opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, q)
    if kernel == "laplace":
        return create_laplace_potential_assembler(OPS[op], opts, dtype or np.float64)
    return create_helmholtz_potential_assembler(OPS[op], k, opts, dtype or np.complex128)


def space(grid, degree):
    return function_space(grid, create_family(
        Family.Lagrange, degree, Continuity.Standard if degree else Continuity.Discontinuous))


def off_surface_points(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * rng.uniform(1.5, 3.0, (n, 1))


@pytest.mark.parametrize("index", range(4))
def test_octahedron_matches_bempp_cl_and_oracle(index):
    from oracle import potential

    with open(os.path.join(os.path.dirname(__file__), "golden",
                           "bempp_cl_octahedron_potentials.json")) as f:
        case = json.load(f)["cases"][index]
    pts, cells = shapes.regular_sphere(0)
    grid = Grid(pts, cells)
    k = case["wavenumber"] or 0.0
    a = assembler(case["kernel"], case["operator"], k)  # default options: 37 points
    p = a.assemble(space(grid, 0), np.array(case["points"]))
    ref = np.array(case["matrix"])
    if ref.ndim == 3:
        ref = ref[..., 0] + 1j * ref[..., 1]
    ref = ref.T  # from_cl[dof][point] -> [point, dof]
    assert np.abs(p - ref).max() <= case["epsilon"]
    o = potential.potential(case["points"], pts, cells, case["kernel"], case["operator"], k=k)
    assert rel_err(p, o) <= FP64_TOL


@pytest.mark.parametrize("degree", [0, 1])
@pytest.mark.parametrize("kernel,op,k", [
    ("laplace", "single_layer", 0.0),
    ("laplace", "double_layer", 0.0),
    ("helmholtz", "single_layer", 5.0),
    ("helmholtz", "double_layer", 5.0),
])
def test_potential_matches_oracle(kernel, op, k, degree):
    from oracle import potential

    pts, cells = shapes.icosphere(3)
    pts = shapes.radial_perturbation(pts, seed=7)
    grid = Grid(pts, cells)
    x = off_surface_points(77, seed=degree)  # 77: a ragged last tile of points
    p = assembler(kernel, op, k, q=6).assemble(space(grid, degree), x)
    o = potential.potential(x, pts, cells, kernel, op, k=k, degree=degree,
                            continuous=bool(degree), q_regular=6)
    assert p.shape == o.shape
    assert rel_err(p, o) <= FP64_TOL


def test_potential_into_device_and_single_precision():
    import torch

    pts, cells = shapes.icosphere(2)
    grid = Grid(pts, cells)
    sp = space(grid, 1)
    x = off_surface_points(40, seed=3)
    a = assembler("helmholtz", "double_layer", 3.0, q=6)
    host = a.assemble(sp, x)
    d_x = torch.as_tensor(x, device="cuda")
    d_out = torch.empty((sp.global_size, x.shape[0]), dtype=torch.complex128, device="cuda")
    a.assemble_into_device(sp, d_x, d_out, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy().T, host) or rel_err(d_out.cpu().numpy().T, host) <= 1e-14
    a32 = assembler("helmholtz", "double_layer", 3.0, q=6, dtype=np.complex64)
    p32 = a32.assemble(sp, x)
    assert p32.dtype == np.complex64
    assert rel_err(p32.astype(np.complex128), host) <= 1e-6


def test_potential_of_other_operators_is_refused():
    with pytest.raises(ValueError):
        create_laplace_potential_assembler(OperatorType.Hypersingular)
