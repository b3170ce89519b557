"""Test shapes as grids (bempp-rs src/shapes.rs; icosphere variants added)."""

from bempp import shapes as _shapes
from ndgrid.grid import Grid


def regular_sphere(level: int) -> Grid:
    return Grid(*_shapes.regular_sphere(level))


def icosphere(level: int) -> Grid:
    return Grid(*_shapes.icosphere(level))
