"""CPU FP64 restatement of the off-surface potential operators (test infrastructure only).

Only the tests import this module; it is the checker for the CUDA potential kernel
(potential.cu) and never part of the product path.

    P[i, j] = sum over the cells c of DOF j of  jdet_c / (4 pi) sum_q w_q psi_b(xi_q) K(x_i, y_c(xi_q))

with K = 1/r (Laplace single layer), (x - y).n_y / r^3 (Laplace double layer),
e^{ikr}/r and e^{ikr}(1 - ikr)(x - y).n_y / r^3 (Helmholtz), r = |x - y|: the kernels of
the reference's boundary operators (src/boundary_assemblers/helpers.rs:7-40,
integrands/single_layer.rs, integrands/double_layer.rs), integrated by the same regular
rule (oracle.simplex_rule) and DOF numbering (oracle.cell_dofs).  The reference has no
evaluator (src/boundary_evaluators.rs is empty); its bempp-cl values for these operators
are the commented tests at tests/compare_to_bempp_cl.rs:208-320, which pin this
restatement to their 1e-3 tolerance (tests/test_oracle_golden.py).  Vectorised numpy,
for small cases (points x cells x rule points x 3 doubles in memory).
"""

from __future__ import annotations

import numpy as np

from . import oracle


def potential(x, points, cells, kernel, operator, *, k=0.0, degree=0, continuous=False,
              q_regular=37):
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    points = np.asarray(points, dtype=np.float64)
    cells = np.asarray(cells, dtype=np.int64)
    xi, w = oracle.simplex_rule(q_regular)
    dofs, n = oracle.cell_dofs(points, cells, degree, continuous)
    v0 = points[cells[:, 0]]
    t0 = points[cells[:, 1]] - v0
    t1 = points[cells[:, 2]] - v0
    cr = np.cross(t0, t1)
    jdet = np.linalg.norm(cr, axis=1)
    nrm = cr / jdet[:, None]
    y = v0[:, None, :] + xi[None, :, 0, None] * t0[:, None, :] + xi[None, :, 1, None] * t1[:, None, :]
    d = x[:, None, None, :] - y[None]                      # [points, cells, q, 3]
    r = np.linalg.norm(d, axis=3)
    if operator == "single_layer":
        kern = 1.0 / r if kernel == "laplace" else np.exp(1j * k * r) / r
    elif operator == "double_layer":
        dn = np.einsum("icqd,cd->icq", d, nrm)
        kern = dn / r ** 3
        if kernel == "helmholtz":
            kern = kern * np.exp(1j * k * r) * (1.0 - 1j * k * r)
    else:
        raise ValueError("potential operators: single_layer and double_layer")
    l0, l1, l2 = 1.0 - xi[:, 0] - xi[:, 1], xi[:, 0], xi[:, 1]
    if degree == 0:
        basis = np.ones((len(w), 1))
    elif degree == 1:
        basis = np.stack([l0, l1, l2], axis=1)
    else:  # nodal P2 basis: vertices, then midpoints of edges [1,2], [0,2], [0,1]
        basis = np.stack([l0 * (2 * l0 - 1), l1 * (2 * l1 - 1), l2 * (2 * l2 - 1),
                          4 * l1 * l2, 4 * l0 * l2, 4 * l0 * l1], axis=1)
    local = np.einsum("icq,q,qb,c->icb", kern, w, basis, jdet) / (4.0 * np.pi)
    out = np.zeros((x.shape[0], n), dtype=local.dtype)
    for b in range(dofs.shape[1]):
        np.add.at(out.T, dofs[:, b], local[:, :, b].T)
    return out
