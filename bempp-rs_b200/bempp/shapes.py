"""Test surfaces: refined octahedron and icosahedron spheres, and seeded deformations.

``regular_sphere`` follows bempp-rs ``shapes::regular_sphere`` (src/shapes.rs:19-114):
start from the unit octahedron (points and cells in the reference's order), then refine
``level`` times; each edge midpoint is created once (in the order cells and their edges
[1,2], [0,2], [0,1] are visited), projected to radius 1, and every cell [c0, c1, c2] is
replaced by [c0, e2, e1], [c1, e0, e2], [c2, e1, e0], [e0, e1, e2] where e_i is the
midpoint of the edge opposite c_i.

``icosphere`` applies the same refinement to a unit icosahedron (12 points, 20
outward-oriented cells), giving 20 * 4**level cells and 10 * 4**level + 2 points
(1,280 / 5,120 / 20,480 cells for levels 3 / 4 / 5).
"""

from __future__ import annotations

import numpy as np


def _refine(points, cells, levels):
    pts = [tuple(p) for p in points]
    cells = [tuple(c) for c in cells]
    for _ in range(levels):
        edge_points = {}
        new_cells = []
        for c in cells:
            mids = []
            for i, j in ((1, 2), (0, 2), (0, 1)):
                a, b = c[i], c[j]
                key = (a, b) if a < b else (b, a)
                idx = edge_points.get(key)
                if idx is None:
                    va, vb = pts[c[i]], pts[c[j]]
                    m = [0.5 * (va[0] + vb[0]), 0.5 * (va[1] + vb[1]), 0.5 * (va[2] + vb[2])]
                    size = np.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])
                    pts.append((m[0] / size, m[1] / size, m[2] / size))
                    idx = len(pts) - 1
                    edge_points[key] = idx
                mids.append(idx)
            e0, e1, e2 = mids
            new_cells += [(c[0], e2, e1), (c[1], e0, e2), (c[2], e1, e0), (e0, e1, e2)]
        cells = new_cells
    return np.array(pts, dtype=np.float64), np.array(cells, dtype=np.int64)


def regular_sphere(level: int):
    """Refined unit octahedron (src/shapes.rs:19-114): 8 * 4**level cells."""
    points = [[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [-1.0, 0.0, 0.0],
              [0.0, -1.0, 0.0], [0.0, 0.0, -1.0]]
    cells = [[0, 1, 2], [0, 2, 3], [0, 3, 4], [0, 4, 1], [5, 2, 1], [5, 3, 2], [5, 4, 3],
             [5, 1, 4]]
    return _refine(points, cells, level)


def _icosahedron():
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    pts = np.array([[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0],
                    [0, -1, phi], [0, 1, phi], [0, -1, -phi], [0, 1, -phi],
                    [phi, 0, -1], [phi, 0, 1], [-phi, 0, -1], [-phi, 0, 1]], dtype=np.float64)
    pts /= np.linalg.norm(pts, axis=1)[:, None]
    cells = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                      [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                      [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                      [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    # orient every cell outward
    for c in cells:
        a, b, d = pts[c[0]], pts[c[1]], pts[c[2]]
        if np.dot(np.cross(b - a, d - a), a + b + d) < 0:
            c[1], c[2] = c[2], c[1]
    return pts, cells


def icosphere(level: int):
    """Refined unit icosahedron: 20 * 4**level cells, 10 * 4**level + 2 points."""
    pts, cells = _icosahedron()
    return _refine(pts, cells, level)


def radial_perturbation(points, seed: int, amplitude: float = 0.02):
    """x_v <- r_v x_v with r_v = 1 + U(-amplitude, amplitude), numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    r = 1.0 + rng.uniform(-amplitude, amplitude, len(points))
    return points * r[:, None]


def ellipsoidal_stretch(points, seed: int, low: float = 0.8, high: float = 1.2):
    """x <- diag(axes) x with axes = U(low, high)^3, numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    axes = rng.uniform(low, high, 3)
    return points * axes[None, :]


def screen_quads(n: int = 3):
    """The flat n x n quadrilateral grid of the unit square in the plane z = 0 (points
    (i/n, j/n, 0), cells [k, k+1, k+n+1, k+n+2] with k = (n+1) j + i: ndelement's vertex
    order), the grid of the reference's quadrilateral assembly cases
    (src/boundary_assemblers.rs:840-865 builds it with n = 3)."""
    pts = np.array([[i / n, j / n, 0.0] for j in range(n + 1) for i in range(n + 1)])
    cells = np.array([[(n + 1) * j + i, (n + 1) * j + i + 1, (n + 1) * (j + 1) + i,
                       (n + 1) * (j + 1) + i + 1] for j in range(n) for i in range(n)],
                     dtype=np.int64)
    return pts, cells


def cube_quads(n: int):
    """Surface of the cube [-1, 1]^3 as 6 n^2 quadrilaterals with shared vertices, in
    ndelement's vertex order (v0, v1 along the first face axis, v2 along the second, v3
    opposite v0) and outward-oriented (first axis x second axis = outward normal)."""
    faces = []  # (origin corner, first axis, second axis), first x second = outward
    for ax in range(3):
        for sgn in (-1.0, 1.0):
            u = [(ax + 1) % 3, (ax + 2) % 3]
            if sgn < 0:
                u = u[::-1]
            o = np.full(3, -1.0)
            o[ax] = sgn
            faces.append((o, u))
    index = {}
    pts = []
    cells = []

    def point(p):
        key = tuple(np.round(p, 12))
        if key not in index:
            index[key] = len(pts)
            pts.append(p)
        return index[key]

    for o, (a, b) in faces:
        for j in range(n):
            for i in range(n):
                def corner(di, dj):
                    p = o.copy()
                    p[a] += 2.0 * (i + di) / n
                    p[b] += 2.0 * (j + dj) / n
                    return point(p)
                cells.append([corner(0, 0), corner(1, 0), corner(0, 1), corner(1, 1)])
    return np.array(pts, dtype=np.float64), np.array(cells, dtype=np.int64)
