"""Flat-triangle surface grid."""

from __future__ import annotations

import numpy as np

from ndelement.reference_cell import ReferenceCellType


class Grid:
    """Triangle grid in 3D: points (npoints x 3) and cells (ncells x 3 point indices)."""

    def __init__(self, points, cells):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.cells = np.ascontiguousarray(cells, dtype=np.uint64)
        if self.points.ndim != 2 or self.points.shape[1] != 3:
            raise ValueError("points must be npoints x 3")
        if self.cells.ndim != 2 or self.cells.shape[1] != 3:
            raise ValueError("cells must be ncells x 3")
        if len(self.cells) and int(self.cells.max()) >= len(self.points):
            raise ValueError("cell vertex index out of range")

    @property
    def topology_dim(self) -> int:
        return 2

    @property
    def geometry_dim(self) -> int:
        return 3

    def entity_count(self, cell: ReferenceCellType) -> int:
        if cell == ReferenceCellType.Point:
            return len(np.unique(self.cells))
        if cell == ReferenceCellType.Interval:
            e = np.sort(self.cells[:, [1, 2, 0, 2, 0, 1]].reshape(-1, 2), axis=1)
            return len(np.unique(e, axis=0))
        if cell == ReferenceCellType.Triangle:
            return len(self.cells)
        return 0
