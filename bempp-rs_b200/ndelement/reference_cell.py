"""Reference cell types (values of ndelement's ReferenceCellType enum)."""

from enum import IntEnum


class ReferenceCellType(IntEnum):
    Point = 0
    Interval = 1
    Triangle = 2
    Quadrilateral = 3
    Tetrahedron = 4
    Hexahedron = 5
    Prism = 6
    Pyramid = 7
