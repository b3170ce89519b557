"""Off-surface potential operators (an addition: the reference declares an evaluator
module, src/boundary_evaluators.rs, that is empty, and keeps its bempp-cl comparisons as
commented tests, tests/compare_to_bempp_cl.rs:208-320).

``PotentialAssembler.assemble(space, points)`` returns the npoints x ndofs matrix
P[i, j] = int psi_j(y) K(x_i, y) dy with K the single-layer kernel G(x, y) or the
double-layer kernel n_y . grad_y G(x, y) of the Laplace or Helmholtz Green's function,
integrated by the regular rule of the options (default 37 points), on the GPU
(``potential_assemble_into_memory`` / ``potential_assemble_into_device`` of the C-ABI).
"""

from __future__ import annotations

import typing

import numpy as np

from bempp._lib import check as _check
from bempp._lib import ffi as _ffi
from bempp._lib import lib as _lib
from bempp.assembly.boundary import (BoundaryAssembler, BoundaryAssemblerOptions, OperatorType,
                                     create_helmholtz_assembler, create_laplace_assembler)
from bempp.function_space import FunctionSpace


class PotentialAssembler(object):
    """Potential assembler: the kernel, operator, dtype and options of a boundary
    assembler, applied between a space and points off the surface."""

    def __init__(self, assembler: BoundaryAssembler, operator_type: OperatorType):
        if operator_type not in (OperatorType.SingleLayer, OperatorType.DoubleLayer):
            raise ValueError("potential operators: single and double layer only")
        self._assembler = assembler
        self.operator_type = operator_type

    @property
    def dtype(self):
        """Data type."""
        return self._assembler.dtype

    def assemble(self, space: FunctionSpace, points) -> np.ndarray:
        """The npoints x ndofs potential matrix for points of shape (npoints, 3)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.empty((pts.shape[0], space.global_size), dtype=self.dtype, order="F")
        _check(
            _lib.potential_assemble_into_memory(
                self._assembler._rs_assembler, space._rs_space,
                _ffi.cast("double*", pts.ctypes.data), pts.shape[0],
                _ffi.cast("void*", out.ctypes.data)),
            "potential assemble",
        )
        return out

    def assemble_into_device(self, space: FunctionSpace, points, out, stream=None):
        """Device variant: ``points`` a CUDA float64 tensor of shape (npoints, 3) (row-major)
        and ``out`` one holding npoints x ndofs elements of the dtype, column-major (a
        tensor of shape (ndofs, npoints)); enqueued on ``stream`` (a cudaStream_t int)."""
        pptr = points.data_ptr() if hasattr(points, "data_ptr") else int(points)
        n = points.shape[0] if hasattr(points, "shape") else None
        if n is None:
            raise ValueError("points must carry a shape (npoints, 3)")
        optr = out.data_ptr() if hasattr(out, "data_ptr") else int(out)
        _check(
            _lib.potential_assemble_into_device(
                self._assembler._rs_assembler, space._rs_space, _ffi.cast("double*", pptr), n,
                _ffi.cast("void*", optr), _ffi.cast("void*", int(stream or 0))),
            "potential assemble_into_device",
        )


def create_laplace_potential_assembler(
    operator_type: OperatorType,
    options: typing.Optional[BoundaryAssemblerOptions] = None,
    dtype: typing.Type[np.floating] = np.float64,
) -> PotentialAssembler:
    """Laplace single- or double-layer potential."""
    return PotentialAssembler(create_laplace_assembler(operator_type, options, dtype), operator_type)


def create_helmholtz_potential_assembler(
    operator_type: OperatorType,
    wavenumber: float,
    options: typing.Optional[BoundaryAssemblerOptions] = None,
    dtype: typing.Type[np.complexfloating] = np.complex128,
) -> PotentialAssembler:
    """Helmholtz single- or double-layer potential."""
    return PotentialAssembler(create_helmholtz_assembler(operator_type, wavenumber, options, dtype),
                              operator_type)
