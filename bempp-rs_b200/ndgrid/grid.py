"""Surface grids of flat triangles or bilinear quadrilaterals."""

from __future__ import annotations

import numpy as np

from ndelement.reference_cell import ReferenceCellType


# local edges of each cell type as ndelement numbers them: a triangle's edge i is opposite
# its vertex i; a quadrilateral's (vertices (0,0), (1,0), (0,1), (1,1)) are [0,1], [0,2],
# [1,3], [2,3]
_EDGES = {3: ((1, 2), (0, 2), (0, 1)), 4: ((0, 1), (0, 2), (1, 3), (2, 3))}


class Grid:
    """Single-element surface grid in 3D: points (npoints x 3) and cells (ncells x 3
    point indices for flat triangles, ncells x 4 for bilinear quadrilaterals with their
    vertices in the reference square's order (0,0), (1,0), (0,1), (1,1)).

    ``cell_vertices`` (optional, same shape as ``cells``) gives the topology's vertex of
    each cell corner when it differs from the point index, as in an ndgrid grid whose
    topology joins coincident points.  Such grids, and every quadrilateral grid, are handed
    to the library through ndgrid's single-element-grid arrays (``topology_arrays``)."""

    def __init__(self, points, cells, cell_vertices=None):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.cells = np.ascontiguousarray(cells, dtype=np.uint64)
        if self.points.ndim != 2 or self.points.shape[1] != 3:
            raise ValueError("points must be npoints x 3")
        if self.cells.ndim != 2 or self.cells.shape[1] not in (3, 4):
            raise ValueError("cells must be ncells x 3 (triangles) or ncells x 4 "
                             "(quadrilaterals)")
        if len(self.cells) and int(self.cells.max()) >= len(self.points):
            raise ValueError("cell vertex index out of range")
        self.cell_vertices = None
        if cell_vertices is not None:
            cv = np.ascontiguousarray(cell_vertices, dtype=np.uint64)
            if cv.shape != self.cells.shape:
                raise ValueError("cell_vertices must have the shape of cells")
            self.cell_vertices = cv

    @property
    def cell_type(self) -> ReferenceCellType:
        """Triangle or Quadrilateral."""
        return (ReferenceCellType.Quadrilateral if self.cells.shape[1] == 4
                else ReferenceCellType.Triangle)

    def topology_arrays(self):
        """ndgrid-style topology of the grid: entity counts per dimension, cell -> vertex
        and cell -> edge connectivity (3 or 4 per cell, ndelement's local edge order) and
        edge -> vertex connectivity (2 per edge).  Vertices are ``cell_vertices`` (or the
        point indices); edges are numbered in first-visit order over the cells and their
        local edges."""
        cv = self.cells if self.cell_vertices is None else self.cell_vertices
        nv = int(cv.max()) + 1 if len(cv) else 0
        index = {}
        cell_edges = np.zeros_like(cv)
        edge_vertices = []
        for c, cell in enumerate(cv.tolist()):
            for i, (la, lb) in enumerate(_EDGES[len(cell)]):
                a, b = cell[la], cell[lb]
                key = (min(a, b), max(a, b))
                e = index.get(key)
                if e is None:
                    e = index[key] = len(edge_vertices)
                    edge_vertices.append(key)
                cell_edges[c, i] = e
        ev = np.array(edge_vertices, dtype=np.uint64).reshape(-1, 2)
        return {"entity_counts": np.array([nv, len(ev), len(cv)], dtype=np.uint64),
                "cell_vertices": np.ascontiguousarray(cv), "cell_edges": cell_edges,
                "edge_vertices": ev}

    @property
    def topology_dim(self) -> int:
        return 2

    @property
    def geometry_dim(self) -> int:
        return 3

    def entity_count(self, cell: ReferenceCellType) -> int:
        if cell == ReferenceCellType.Point:
            cv = self.cells if self.cell_vertices is None else self.cell_vertices
            return len(np.unique(cv))
        if cell == ReferenceCellType.Interval:
            cv = self.cells if self.cell_vertices is None else self.cell_vertices
            local = [v for edge in _EDGES[cv.shape[1]] for v in edge]
            e = np.sort(cv[:, local].reshape(-1, 2), axis=1)
            return len(np.unique(e, axis=0))
        if cell == self.cell_type:
            return len(self.cells)
        return 0
