"""CPU restatement of the reference's QP adjoint derivative path (float64).

TEST INFRASTRUCTURE ONLY (oracle).

Restates ``warpmpc/jax_osqp/solver.py``:

* ``_build_derivative_plan`` 413-571: inequality rows split into lower
  (``G = -A_r``, ``h = -l_r``) and upper (``G = A_r``, ``h = u_r``) parts
  for finite bounds with ``l < u``; equality rows ``l == u``;
* ``_adjoint_derivative_compute_jit`` 1084-1156: with ``y_u = max(y, 0)``,
  ``y_l = -min(y, 0)``, slacks ``s = G x - h``, the matrix
  ``M = [[P, G^T diag(lambda), Aeq^T], [G, diag(s), 0], [Aeq, 0, 0]]`` (the
  transposed KKT Jacobian) inside the quasi-definite augmented system
  ``[[(1+eps) I, M], [M^T, -eps I]]`` (eps = 1e-6), right-hand side
  ``-[dx; dy_l; dy_u; d_nu]``, solved here densely and exactly, followed by
  the reference's iterative refinement against the unperturbed matrix;
* ``_adjoint_derivative_get_vec`` / ``_get_mat`` 1158-1192: ``dq = rx``,
  ``dl = ryl``, ``du = -ryu``, ``dP`` on P's upper pattern,
  ``dA = (y_u - y_l) rx^T + (ryu - ryl) x^T`` on A's pattern.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg

OSQP_INFTY = 1e30
OSQP_MIN_SCALING = 1e-4


def adjoint(plan, p_values, a_values, l, u, x, y, dx, dy, eps=1e-6, refinement_iters=100):
    """One instance (1-D arrays).  Returns (dq, dl, du, dP_upper, dA)."""
    n, m = plan.n, plan.m
    p_rows = plan.p_upper.indices
    p_cols = np.repeat(np.arange(n), np.diff(plan.p_upper.indptr))
    a_rows, a_cols = plan.a_rows, plan.a_cols
    P = np.zeros((n, n))
    P[p_rows, p_cols] = p_values
    P = P + np.triu(P, 1).T
    A = np.zeros((m, n))
    A[a_rows, a_cols] = a_values
    infval = OSQP_INFTY * OSQP_MIN_SCALING
    is_ineq = l < u
    lower = np.flatnonzero(is_ineq & (l > -infval))
    upper = np.flatnonzero(is_ineq & (u < infval))
    eq = np.flatnonzero(~is_ineq)
    G = np.vstack([-A[lower], A[upper]])
    h = np.concatenate([-l[lower], u[upper]])
    Aeq = A[eq]
    y_u = np.maximum(y, 0.0)
    y_l = -np.minimum(y, 0.0)
    lam = np.concatenate([y_l[lower], y_u[upper]])
    s = G @ x - h
    ni, ne = G.shape[0], Aeq.shape[0]
    half = n + ni + ne
    M = np.zeros((half, half))
    M[:n, :n] = P
    M[:n, n : n + ni] = G.T * lam[None, :]
    M[:n, n + ni :] = Aeq.T
    M[n : n + ni, :n] = G
    M[n : n + ni, n : n + ni] = np.diag(s)
    M[n + ni :, :n] = Aeq
    K0 = np.block([[np.eye(half), M], [M.T, np.zeros((half, half))]])
    K = np.block([[(1.0 + eps) * np.eye(half), M], [M.T, -eps * np.eye(half)]])
    rhs = np.zeros(2 * half)
    rhs[:n] = -dx
    rhs[n : n + lower.size] = -dy[lower]
    rhs[n + lower.size : n + ni] = -dy[upper]
    d_nu = np.where(y[eq] >= 0.0, dy[eq], -dy[eq])
    rhs[n + ni : half] = -d_nu
    lu = scipy.linalg.lu_factor(K)  # one factorization, reused by every refinement solve
    sol = scipy.linalg.lu_solve(lu, rhs)
    for _ in range(refinement_iters):
        sol = sol - scipy.linalg.lu_solve(lu, K0 @ sol - rhs)
    rx = sol[half : half + n]
    r_yl = np.zeros(m)
    r_yu = np.zeros(m)
    pos = half + n
    r_yl[lower] = -sol[pos : pos + lower.size]
    pos += lower.size
    r_yu[upper] = sol[pos : pos + upper.size]
    pos += upper.size
    eq_sol = sol[pos : pos + ne]
    eq_y = y[eq]
    with np.errstate(divide="ignore", invalid="ignore"):
        r_yu[eq] = np.where(eq_y >= 0.0, eq_sol / eq_y, 0.0)
        r_yl[eq] = np.where(eq_y >= 0.0, 0.0, -eq_sol / eq_y)
    ryl = -(r_yl * y_l)
    ryu = r_yu * y_u
    dP = 0.5 * (rx[p_rows] * x[p_cols] + rx[p_cols] * x[p_rows])
    dA = (y_u - y_l)[a_rows] * rx[a_cols] + (ryu - ryl)[a_rows] * x[a_cols]
    return rx, ryl, -ryu, dP, dA


def active_set_adjoint(plan, p_values, a_values, l, u, x, z, y, dx, dy):
    """Exact derivative of the QP solution on the active set (float64).

    Active rows: equality rows (l == u, side by the sign of y) and rows whose
    projected value z sits on a bound.  Solves
    ``[[P, A_C^T], [A_C, 0]] [w; mu] = [-dx; -tau dy_C]`` densely and returns
    the reference's outputs (dq, dl, du, dP_upper, dA) for that solution.  It
    is the limit the reference's regularized path converges to on
    non-degenerate problems, and is checked against central finite
    differences in the tests.
    """
    n, m = plan.n, plan.m
    p_rows = plan.p_upper.indices
    p_cols = np.repeat(np.arange(n), np.diff(plan.p_upper.indptr))
    P = np.zeros((n, n))
    P[p_rows, p_cols] = p_values
    P = P + np.triu(P, 1).T
    A = np.zeros((m, n))
    A[plan.a_rows, plan.a_cols] = a_values
    tau = np.zeros(m, dtype=int)
    eq = l == u
    tau[eq] = np.where(y[eq] >= 0, 1, -1)
    tau[~eq & (z >= u)] = 1
    tau[~eq & (z < u) & (z <= l)] = -1
    C = np.flatnonzero(tau != 0)
    K = np.block([[P, A[C].T], [A[C], np.zeros((C.size, C.size))]])
    sol = np.linalg.lstsq(K, np.concatenate([-dx, -tau[C] * dy[C]]), rcond=None)[0]
    w = sol[:n]
    mu = np.zeros(m)
    mu[C] = sol[n:]
    dl = np.where(tau < 0, -mu, 0.0)
    du = np.where(tau > 0, -mu, 0.0)
    dP = 0.5 * (w[p_rows] * x[p_cols] + w[p_cols] * x[p_rows])
    nu = np.where(tau != 0, mu, 0.0)
    dA = y[plan.a_rows] * w[plan.a_cols] + nu[plan.a_rows] * x[plan.a_cols]
    return w, dl, du, dP, dA
