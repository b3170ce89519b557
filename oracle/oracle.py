"""ctypes front end of the CPU FP64 oracle (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this module; it is the checker for the CUDA assembler and never part of the
product path.  The library is built on demand by ``make`` for the CPU it runs on
(``-march=native``), keyed by a hash of the CPU's model name and flags.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_lib = None

OPERATORS = {"single_layer": 0, "double_layer": 1, "adjoint_double_layer": 2,
             "hypersingular": 3}


def _cpu_tag() -> str:
    info = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.strip() == "":
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:10]


def library_path() -> str:
    return os.path.join(_HERE, f"liboracle_{_cpu_tag()}.so")


def build() -> str:
    path = library_path()
    tag = os.path.basename(path)[len("liboracle_"):-3]
    subprocess.run(["make", "-s", "-C", _HERE, f"TAG={tag}"], check=True)
    return path


def lib():
    global _lib
    with _lock:
        if _lib is None:
            path = build()
            L = ctypes.CDLL(path)
            i64p = ctypes.POINTER(ctypes.c_int64)
            dp = ctypes.POINTER(ctypes.c_double)
            L.oracle_assemble_dense.restype = ctypes.c_int
            L.oracle_assemble_dense.argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int64, i64p,
                ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, i64p,
                ctypes.c_int64, ctypes.c_void_p]
            L.oracle_last_error.restype = ctypes.c_char_p
            L.oracle_cell_dofs.restype = ctypes.c_int64
            L.oracle_cell_dofs.argtypes = [i64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_int, i64p]
            L.oracle_colouring.restype = ctypes.c_int
            L.oracle_colouring.argtypes = [i64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_int32)]
            L.oracle_duffy_rule.restype = ctypes.c_int
            L.oracle_duffy_rule.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
            L.oracle_simplex_rule.restype = ctypes.c_int
            L.oracle_simplex_rule.argtypes = [ctypes.c_int, dp, dp]
            L.oracle_quad_assemble_dense.restype = ctypes.c_int
            L.oracle_quad_assemble_dense.argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int64, i64p,
                ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
            L.oracle_quad_last_error.restype = ctypes.c_char_p
            L.oracle_quad_cell_dofs.restype = ctypes.c_int64
            L.oracle_quad_cell_dofs.argtypes = [i64p, ctypes.c_int64, ctypes.c_int64,
                                                ctypes.c_int, ctypes.c_int, i64p]
            L.oracle_quad_duffy_rule.restype = ctypes.c_int
            L.oracle_quad_duffy_rule.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
            _lib = L
    return _lib


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def nbasis(degree):
    return {0: 1, 1: 3, 2: 6}[degree]


def space_size(points, cells, degree, continuous):
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    out = np.empty(cells.shape[0] * nbasis(degree), dtype=np.int64)
    return int(lib().oracle_cell_dofs(_ptr(cells, ctypes.c_int64), cells.shape[0],
                                      len(points), degree, int(continuous),
                                      _ptr(out, ctypes.c_int64)))


def cell_dofs(points, cells, degree, continuous):
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    nb = nbasis(degree)
    out = np.empty(cells.shape[0] * nb, dtype=np.int64)
    n = lib().oracle_cell_dofs(_ptr(cells, ctypes.c_int64), cells.shape[0], len(points),
                               degree, int(continuous), _ptr(out, ctypes.c_int64))
    return out.reshape(-1, nb), int(n)


def colouring(points, cells, degree, continuous):
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    out = np.empty(cells.shape[0], dtype=np.int32)
    n = lib().oracle_colouring(_ptr(cells, ctypes.c_int64), cells.shape[0], len(points),
                               degree, int(continuous), _ptr(out, ctypes.c_int32))
    return out, int(n)


def duffy_rule(config, order):
    L = lib()
    n = L.oracle_duffy_rule(config, order, None, None, None)
    tp = np.empty(2 * n)
    sp = np.empty(2 * n)
    w = np.empty(n)
    L.oracle_duffy_rule(config, order, _ptr(tp, ctypes.c_double), _ptr(sp, ctypes.c_double),
                        _ptr(w, ctypes.c_double))
    return tp.reshape(n, 2), sp.reshape(n, 2), w


def simplex_rule(npoints):
    L = lib()
    pts = np.empty(2 * npoints)
    wts = np.empty(npoints)
    if L.oracle_simplex_rule(npoints, _ptr(pts, ctypes.c_double), _ptr(wts, ctypes.c_double)) < 0:
        raise ValueError(f"no rule with {npoints} points")
    return pts.reshape(npoints, 2), wts


def assemble(points, cells, kernel, operator, *, k=0.0, test_degree=0, test_continuous=False,
             trial_degree=0, trial_continuous=False, q_regular=37, q_singular=4,
             batch_size=128, nthreads=0, parts=3, test_subset=None):
    """Dense FP64 matrix (n_test x n_trial, Fortran order) of a Laplace or Helmholtz
    boundary operator, assembled on the CPU exactly as bempp-rs structures it."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    helm = kernel == "helmholtz"
    n_test = space_size(points, cells, test_degree, test_continuous)
    n_trial = space_size(points, cells, trial_degree, trial_continuous)
    out = np.zeros((n_test, n_trial), dtype=np.complex128 if helm else np.float64, order="F")
    subset = None
    nsub = 0
    if test_subset is not None:
        subset = np.ascontiguousarray(test_subset, dtype=np.int64)
        nsub = len(subset)
    rc = lib().oracle_assemble_dense(
        int(helm), OPERATORS[operator], float(k), _ptr(points, ctypes.c_double), len(points),
        _ptr(cells, ctypes.c_int64), cells.shape[0], test_degree, int(test_continuous),
        trial_degree, int(trial_continuous), q_regular, q_singular, batch_size, nthreads, parts,
        _ptr(subset, ctypes.c_int64) if subset is not None else None, nsub,
        out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError(lib().oracle_last_error().decode())
    return out


# ------------------------------------------------------------ quadrilateral grids ---
def quad_cell_dofs(points, cells, degree, continuous):
    """DOF map of a Lagrange degree-0 / 1 space on a quadrilateral grid (ncells x 4)."""
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    nb = 1 if degree == 0 else 4
    out = np.empty(cells.shape[0] * nb, dtype=np.int64)
    n = lib().oracle_quad_cell_dofs(_ptr(cells, ctypes.c_int64), cells.shape[0], len(points),
                                    degree, int(continuous), _ptr(out, ctypes.c_int64))
    return out.reshape(-1, nb), int(n)


def quad_duffy_rule(config, order):
    L = lib()
    n = L.oracle_quad_duffy_rule(config, order, None, None, None)
    tp = np.empty(2 * n)
    sp = np.empty(2 * n)
    w = np.empty(n)
    L.oracle_quad_duffy_rule(config, order, _ptr(tp, ctypes.c_double), _ptr(sp, ctypes.c_double),
                             _ptr(w, ctypes.c_double))
    return tp.reshape(n, 2), sp.reshape(n, 2), w


def quad_assemble(points, cells, kernel, operator, *, k=0.0, test_degree=0,
                  test_continuous=False, trial_degree=0, trial_continuous=False, q_regular=16,
                  q_singular=4, nthreads=0, parts=3):
    """Dense FP64 matrix of a boundary operator on a quadrilateral grid (ncells x 4 cells in
    ndelement's vertex order), Gauss tensor regular rule of n x n points, n the smallest
    with n^2 >= q_regular."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    cells = np.ascontiguousarray(cells, dtype=np.int64)
    helm = kernel == "helmholtz"
    _, n_test = quad_cell_dofs(points, cells, test_degree, test_continuous)
    _, n_trial = quad_cell_dofs(points, cells, trial_degree, trial_continuous)
    out = np.zeros((n_test, n_trial), dtype=np.complex128 if helm else np.float64, order="F")
    rc = lib().oracle_quad_assemble_dense(
        int(helm), OPERATORS[operator], float(k), _ptr(points, ctypes.c_double), len(points),
        _ptr(cells, ctypes.c_int64), cells.shape[0], test_degree, int(test_continuous),
        trial_degree, int(trial_continuous), q_regular, q_singular, nthreads, parts,
        out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError(lib().oracle_quad_last_error().decode())
    return out
