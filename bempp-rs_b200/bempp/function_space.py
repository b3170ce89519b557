"""Function space.

Mirrors python/bempp/function_space.py of bempp-rs: ``function_space(grid, family)``
returns a ``FunctionSpace`` wrapping the library's SpaceT handle, with the same methods
and properties.  The grid is handed to the library once per grid object
(``bempp_grid_from_points_cells``) and shared by every space on it, so spaces built on
the same grid object share one GridT handle, which is what makes the assembler treat
test and trial spaces as living on the same grid (pointer equality, as bempp-rs
``equal_grids``).
"""

from __future__ import annotations

import typing

import numpy as np

from bempp._lib import ffi as _ffi
from bempp._lib import lib as _lib
from ndelement.ciarlet import CiarletElement, ElementFamily
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

_dtypes = {
    _lib.DType_F32: np.float32,
    _lib.DType_F64: np.float64,
    _lib.DType_C32: np.complex64,
    _lib.DType_C64: np.complex128,
}
_rtypes = {v: k for k, v in _dtypes.items()}


class FunctionSpace(object):
    """Function space."""

    def __init__(self, grid: Grid, family: ElementFamily, rs_space, owned: bool = True):
        """Initialise."""
        if rs_space == _ffi.NULL:
            raise ValueError(_ffi.string(_lib.bempp_last_error()).decode())
        self._rs_space = rs_space
        self._owned = owned
        self._grid = grid
        self._family = family

    def __del__(self):
        """Delete."""
        if getattr(self, "_owned", False):
            _lib.space_t_free(self._rs_space)
            self._family._bempp_rs_family_refcount -= 1
            if self._family._bempp_rs_family_refcount == 0:
                _lib.element_family_t_free_bempp(self._family._bempp_rs_family)
                del self._family._bempp_rs_family
                del self._family._bempp_rs_family_refcount
            self._grid._bempp_rs_grid_refcount -= 1
            if self._grid._bempp_rs_grid_refcount == 0:
                _lib.grid_t_free_bempp(self._grid._bempp_rs_grid)
                del self._grid._bempp_rs_grid

    def element(self, entity: ReferenceCellType) -> CiarletElement:
        """Get the element on a cell type."""
        return self._family.element(entity)

    def get_local_dof_numbers(self, entity_dim: int, entity_index: int) -> typing.List[int]:
        """Get the local DOF numbers associated with an entity."""
        dofs = np.empty(
            _lib.space_get_local_dof_numbers_size(self._rs_space, entity_dim, entity_index),
            dtype=np.uintp,
        )
        _lib.space_get_local_dof_numbers(
            self._rs_space, entity_dim, entity_index, _ffi.cast("uintptr_t*", dofs.ctypes.data)
        )
        return [int(i) for i in dofs]

    def cell_dofs(self, cell: int) -> typing.Optional[typing.List[int]]:
        """Get the local DOF numbers associated with a cell."""
        if not _lib.space_has_cell_dofs(self._rs_space, cell):
            return None
        dofs = np.empty(_lib.space_cell_dofs_size(self._rs_space, cell), dtype=np.uintp)
        _lib.space_cell_dofs(self._rs_space, cell, _ffi.cast("uintptr_t*", dofs.ctypes.data))
        return [int(i) for i in dofs]

    def global_dof_index(self, local_dof_index: int) -> int:
        """Get the global DOF number for a local DOF."""
        return _lib.space_global_dof_index(self._rs_space, local_dof_index)

    def ownership(self, local_dof_index):
        """The owning process and index of a local DOF (serial spaces own every DOF)."""
        if _lib.space_is_owned(self._rs_space, local_dof_index):
            return ("owned",)
        return ("ghost", _lib.space_ownership_process(self._rs_space, local_dof_index),
                _lib.space_ownership_index(self._rs_space, local_dof_index))

    @property
    def dtype(self):
        """Data type."""
        return _dtypes[_lib.space_dtype(self._rs_space)]

    @property
    def local_size(self) -> int:
        """Number of DOFs on current process."""
        return _lib.space_local_size(self._rs_space)

    @property
    def global_size(self) -> int:
        """Number of DOFs on all processes."""
        return _lib.space_global_size(self._rs_space)

    @property
    def is_serial(self) -> bool:
        """Indicates whether the function space is stored in serial."""
        return _lib.space_is_serial(self._rs_space)

    @property
    def grid(self) -> Grid:
        """Get the grid that this space is defined on."""
        return self._grid


def function_space(grid: Grid, family: ElementFamily) -> FunctionSpace:
    """Create a function space."""
    if not hasattr(grid, "_bempp_rs_grid"):
        grid._bempp_rs_grid = recreate_grid(grid)
        grid._bempp_rs_grid_refcount = 0
    grid._bempp_rs_grid_refcount += 1
    if not hasattr(family, "_bempp_rs_family"):
        family._bempp_rs_family = recreate_element_family(family)
        family._bempp_rs_family_refcount = 0
    family._bempp_rs_family_refcount += 1
    return FunctionSpace(
        grid, family, _lib.function_space(grid._bempp_rs_grid, family._bempp_rs_family)
    )


def recreate_element_family(family: ElementFamily):
    fam = _lib.create_lagrange_family_bempp(
        family.degree, int(family.continuity), _rtypes[np.dtype(family.dtype).type]
    )
    if fam == _ffi.NULL:
        raise ValueError(_ffi.string(_lib.bempp_last_error()).decode())
    return fam


def recreate_grid(grid: Grid):
    points = np.ascontiguousarray(grid.points, dtype=np.float64)
    cells = np.ascontiguousarray(grid.cells, dtype=np.uintp)
    g = _lib.bempp_grid_from_points_cells(
        _ffi.cast("void*", points.ctypes.data), len(points), _lib.DType_F64,
        _ffi.cast("size_t*", cells.ctypes.data), len(cells))
    if g == _ffi.NULL:
        raise ValueError(_ffi.string(_lib.bempp_last_error()).decode())
    return g
