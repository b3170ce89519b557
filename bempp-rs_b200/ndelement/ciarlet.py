"""Element families (the subset of ndelement.ciarlet that bempp's binding uses)."""

from __future__ import annotations

from enum import Enum, IntEnum

import numpy as np

from ndelement.reference_cell import ReferenceCellType


class Family(Enum):
    Lagrange = 0
    RaviartThomas = 1
    NedelecFirstKind = 2


class Continuity(IntEnum):
    Standard = 0
    Discontinuous = 1


class CiarletElement:
    """Lagrange element on a triangle: degree 0 (one DOF), 1 (three) or 2 (six: the
    vertices, then the midpoints of edges [1,2], [0,2], [0,1]); on a quadrilateral:
    degree 0 (one DOF) or 1 (four, one per vertex)."""

    def __init__(self, cell: ReferenceCellType, degree: int, continuity: Continuity):
        self.cell_type = cell
        self.degree = degree
        self.continuity = continuity

    @property
    def dim(self) -> int:
        if self.cell_type == ReferenceCellType.Quadrilateral:
            return {0: 1, 1: 4, 2: 9}[self.degree]
        return {0: 1, 1: 3, 2: 6}[self.degree]


class ElementFamily:
    def __init__(self, family: Family, degree: int, continuity: Continuity, dtype=np.float64):
        self.family = family
        self.degree = degree
        self.continuity = continuity
        self.dtype = dtype

    def element(self, cell: ReferenceCellType) -> CiarletElement:
        return CiarletElement(cell, self.degree, self.continuity)


def create_family(family: Family, degree: int, continuity: Continuity = Continuity.Standard,
                  dtype=np.float64) -> ElementFamily:
    if family != Family.Lagrange:
        raise ValueError(f"{family} is not supported by the dense assembler")
    if degree == 0:
        continuity = Continuity.Discontinuous
    return ElementFamily(family, degree, continuity, dtype)
