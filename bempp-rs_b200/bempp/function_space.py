"""Function spaces on a grid: the Python face of the library's SpaceT handles.

``function_space(grid, family)`` keeps the call signature and the ``FunctionSpace``
methods of bempp-rs's ``python/bempp/function_space.py`` (those are the API a user
switching from the reference calls).  The handle bookkeeping underneath is this
package's own:

* every native handle (grid, element family, space) is owned by one ``_Owned`` object
  whose ``weakref.finalize`` releases it exactly once, when the last Python reference to
  the owner disappears, or at interpreter exit;
* a grid object is uploaded once: ``grid_handle(grid)`` remembers its owner in a
  ``WeakKeyDictionary`` keyed by the grid object, so every space built on one grid object
  shares one GridT (the library treats test and trial spaces as one grid exactly when the
  GridT pointers agree, as bempp-rs's ``equal_grids`` compares pointers);
* a space's owner keeps the owners of its grid and family alive, so a GridT is released
  only after every space on it, whatever order Python collects the objects in.

Other modules that need a GridT for a grid object (the batched sweep) use
``grid_handle`` too and hold the returned owner while they use it.
"""

from __future__ import annotations

import typing
import weakref

import numpy as np

from bempp._lib import ffi as _ffi
from bempp._lib import last_error as _last_error
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


class _Owned:
    """One native handle and the function that releases it.

    ``keep`` lists other owners this handle depends on; the finalizer holds them, so they
    are released after this one."""

    __slots__ = ("ptr", "_release", "__weakref__")

    def __init__(self, ptr, free, keep=()):
        if ptr == _ffi.NULL:
            raise ValueError(_last_error())
        self.ptr = ptr
        self._release = weakref.finalize(self, _release_handle, free, ptr, tuple(keep))

    def release(self):
        """Release the handle now (idempotent)."""
        self._release()


def _release_handle(free, ptr, keep):
    try:
        free(ptr)
    except Exception:  # the library may already be unloaded at interpreter exit
        pass
    del keep  # dependencies go after the handle that used them


_grid_owners: "weakref.WeakKeyDictionary[Grid, _Owned]" = weakref.WeakKeyDictionary()
_family_owners: "weakref.WeakKeyDictionary[ElementFamily, _Owned]" = weakref.WeakKeyDictionary()


def grid_handle(grid: Grid) -> _Owned:
    """The owner of ``grid``'s GridT, uploading the grid on first use."""
    owner = _grid_owners.get(grid)
    if owner is None:
        owner = _Owned(recreate_grid(grid), _lib.grid_t_free_bempp)
        _grid_owners[grid] = owner
    return owner


def family_handle(family: ElementFamily) -> _Owned:
    """The owner of ``family``'s ElementFamilyT, created on first use."""
    owner = _family_owners.get(family)
    if owner is None:
        owner = _Owned(recreate_element_family(family), _lib.element_family_t_free_bempp)
        _family_owners[family] = owner
    return owner


class FunctionSpace(object):
    """A discrete function space (DOF numbering of a Lagrange family on a grid)."""

    def __init__(self, grid: Grid, family: ElementFamily, rs_space, owned: bool = True):
        """Wrap a SpaceT handle; ``owned`` spaces release it when collected."""
        if rs_space == _ffi.NULL:
            raise ValueError(_last_error())
        self._grid = grid
        self._family = family
        self._rs_space = rs_space
        self._owner = None
        if owned:
            deps = (grid_handle(grid), family_handle(family))
            self._owner = _Owned(rs_space, _lib.space_t_free, keep=deps)

    def element(self, entity: ReferenceCellType) -> CiarletElement:
        """The family's element on cells of type ``entity``."""
        return self._family.element(entity)

    def get_local_dof_numbers(self, entity_dim: int, entity_index: int) -> typing.List[int]:
        """Local DOF numbers attached to entity ``entity_index`` of dimension ``entity_dim``."""
        n = _lib.space_get_local_dof_numbers_size(self._rs_space, entity_dim, entity_index)
        dofs = np.empty(n, dtype=np.uintp)
        _lib.space_get_local_dof_numbers(
            self._rs_space, entity_dim, entity_index, _ffi.cast("uintptr_t*", dofs.ctypes.data)
        )
        return dofs.tolist()

    def cell_dofs(self, cell: int) -> typing.Optional[typing.List[int]]:
        """Local DOF numbers of one cell in its element's order, or None for a cell this
        process does not hold."""
        if not _lib.space_has_cell_dofs(self._rs_space, cell):
            return None
        dofs = np.empty(_lib.space_cell_dofs_size(self._rs_space, cell), dtype=np.uintp)
        _lib.space_cell_dofs(self._rs_space, cell, _ffi.cast("uintptr_t*", dofs.ctypes.data))
        return dofs.tolist()

    def cell_colouring(self) -> typing.Dict[ReferenceCellType, typing.List[typing.List[int]]]:
        """Cells grouped so that no two cells of a group share a DOF entity (the
        reference's FunctionSpace::cell_colouring): {cell type: [cells of colour 0, ...]}."""
        ncells = len(self._grid.cells)
        colours = np.zeros(ncells, dtype=np.uintp)
        n = _lib.space_cell_colouring(self._rs_space, _ffi.cast("size_t*", colours.ctypes.data))
        groups: typing.List[typing.List[int]] = [[] for _ in range(n)]
        for cell, c in enumerate(colours.tolist()):
            groups[c].append(cell)
        return {self._grid.cell_type: groups}

    def global_dof_index(self, local_dof_index: int) -> int:
        """Global number of a local DOF (the identity for serial spaces)."""
        return _lib.space_global_dof_index(self._rs_space, local_dof_index)

    def ownership(self, local_dof_index):
        """("owned",) for a DOF this process owns, else ("ghost", process, index)."""
        if _lib.space_is_owned(self._rs_space, local_dof_index):
            return ("owned",)
        return ("ghost", _lib.space_ownership_process(self._rs_space, local_dof_index),
                _lib.space_ownership_index(self._rs_space, local_dof_index))

    @property
    def dtype(self):
        """Scalar type of the space's family."""
        return _dtypes[_lib.space_dtype(self._rs_space)]

    @property
    def local_size(self) -> int:
        """DOFs held by this process."""
        return _lib.space_local_size(self._rs_space)

    @property
    def global_size(self) -> int:
        """DOFs over all processes (equal to local_size for serial spaces)."""
        return _lib.space_global_size(self._rs_space)

    @property
    def is_serial(self) -> bool:
        """True when one process holds the whole space (always, in this library)."""
        return _lib.space_is_serial(self._rs_space)

    @property
    def grid(self) -> Grid:
        """The grid object the space was built on."""
        return self._grid


def function_space(grid: Grid, family: ElementFamily) -> FunctionSpace:
    """Build the space of ``family`` on ``grid`` (spaces on one grid object share its
    uploaded GridT)."""
    gh = grid_handle(grid)
    fh = family_handle(family)
    return FunctionSpace(grid, family, _lib.function_space(gh.ptr, fh.ptr))


def recreate_element_family(family: ElementFamily):
    """A new ElementFamilyT for a Lagrange family (caller owns it)."""
    fam = _lib.create_lagrange_family_bempp(
        family.degree, int(family.continuity), _rtypes[np.dtype(family.dtype).type]
    )
    if fam == _ffi.NULL:
        raise ValueError(_last_error())
    return fam


def recreate_grid(grid: Grid):
    """A new GridT holding a copy of ``grid`` (caller owns it).  A grid with its own
    topology goes through ndgrid's single-element-grid arrays
    (single_element_grid_borrowed_create_bempp), so that its vertex and edge numbering
    are the ones the library uses; otherwise points and cells suffice."""
    points = np.ascontiguousarray(grid.points, dtype=np.float64)
    cells = np.ascontiguousarray(grid.cells, dtype=np.uintp)
    if getattr(grid, "cell_vertices", None) is None and cells.shape[1] == 3:
        g = _lib.bempp_grid_from_points_cells(
            _ffi.cast("void*", points.ctypes.data), len(points), _lib.DType_F64,
            _ffi.cast("size_t*", cells.ctypes.data), len(cells))
    else:
        g = _ndgrid_create(grid, points, cells)
    if g == _ffi.NULL:
        raise ValueError(_last_error())
    return g


def _ndgrid_create(grid: Grid, points, cells):
    """Call single_element_grid_borrowed_create_bempp with ndgrid-shaped arrays."""
    t = grid.topology_arrays()
    counts = np.ascontiguousarray(t["entity_counts"], dtype=np.uintp)
    cv = np.ascontiguousarray(t["cell_vertices"], dtype=np.uintp)
    ce = np.ascontiguousarray(t["cell_edges"], dtype=np.uintp)
    ev = np.ascontiguousarray(t["edge_vertices"], dtype=np.uintp)
    keep = [counts, cv, ce, ev]  # alive until the library has copied them

    def ptr(a):
        return _ffi.cast("size_t*", a.ctypes.data)

    # downward_connectivity[d][sd]: per entity of dimension d its sub-entities of
    # dimension sd; only the three arrays the library reads are filled in
    d0 = _ffi.new("size_t*[1]", [_ffi.NULL])
    d1 = _ffi.new("size_t*[2]", [ptr(ev), _ffi.NULL])
    d2 = _ffi.new("size_t*[3]", [ptr(cv), ptr(ce), _ffi.NULL])
    down = _ffi.new("size_t**[3]", [d0, d1, d2])
    nvc = cells.shape[1]  # 3 (triangles) or 4 (quadrilaterals)
    s0 = _ffi.new("size_t[1]", [1])
    s1 = _ffi.new("size_t[2]", [2, 1])
    s2 = _ffi.new("size_t[3]", [nvc, nvc, 1])
    shape0 = _ffi.new("size_t*[3]", [s0, s1, s2])
    types = _ffi.new("ReferenceCellType[3]", [
        _lib.ReferenceCellType_Point, _lib.ReferenceCellType_Interval,
        _lib.ReferenceCellType_Quadrilateral if nvc == 4 else _lib.ReferenceCellType_Triangle])
    g = _lib.single_element_grid_borrowed_create_bempp(
        2, _ffi.NULL, _ffi.NULL, types, ptr(counts), down, shape0, _ffi.NULL, _ffi.NULL,
        _ffi.cast("void*", points.ctypes.data), 3, len(points), _lib.DType_F64, ptr(cells),
        nvc, len(cells), 1)
    del keep
    return g
