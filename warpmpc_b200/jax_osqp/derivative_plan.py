"""Pattern of the reference-style adjoint KKT system (``build_osqp_plan(..., derivatives=True)``).

Restates ``_build_derivative_plan`` (``warpmpc/jax_osqp/solver.py:413-571``)
with its helpers ``_full_symmetric_csc_pattern`` (346-374) and
``_selected_a_csc_pattern`` (377-410): the same index arrays in the same
orders, built with sorts instead of per-entry dictionaries.

The system is the quasi-definite augmented matrix
``[[(1 + eps) I, M], [M^T, -eps I]]`` of dimension ``2 (n + n_ineq + n_eq)``
(upper triangle stored), where ``M = [[P, G^T diag(lambda), Aeq^T],
[G, diag(s), 0], [Aeq, 0, 0]]``: inequality rows with a finite lower bound
enter G negated, rows with a finite upper bound as they are, equality rows
(``l == u``) form Aeq.  The numeric data stored with the pattern uses the
representative P and A values (lambda = 0, slack diagonal -1), as the
reference's does; a solve rewrites it per instance through the ``*_pos``
position arrays.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from ..jax_qdldl.planning import build_qdldl_plan
from .types import OSQPDerivativePlan

OSQP_INFTY = 1e30
OSQP_MIN_SCALING = 1e-4
ADJOINT_EPS = 1e-6


def _entries(matrix: sp.csc_matrix):
    """(rows, cols, storage positions) of a CSC matrix in storage order."""
    cols = np.repeat(np.arange(matrix.shape[1], dtype=np.int64), np.diff(matrix.indptr))
    return matrix.indices.astype(np.int64), cols, np.arange(matrix.indices.size, dtype=np.int64)


def _csc_order(rows, cols):
    """Permutation putting (row, col) entries in CSC order (by column, then row)."""
    return np.lexsort((rows, cols))


def full_symmetric_pattern(p_upper: sp.csc_matrix):
    """Both triangles of P in CSC order with the upper entry each one reads
    (solver.py:346-374).  Returns (rows, cols, value_map), int32."""
    r, c, ptr = _entries(p_upper)
    off = r != c
    rows = np.concatenate([r, c[off]])
    cols = np.concatenate([c, r[off]])
    vmap = np.concatenate([ptr, ptr[off]])
    o = _csc_order(rows, cols)
    return rows[o].astype(np.int32), cols[o].astype(np.int32), vmap[o].astype(np.int32)


def selected_rows_pattern(a_matrix: sp.csc_matrix, selected: np.ndarray, row_offset: int = 0):
    """A's entries in the selected rows, renumbered ``row_offset + position in
    selected``, in CSC order (solver.py:377-410).  Returns (rows, cols, a_ptr)."""
    r, c, ptr = _entries(a_matrix)
    where = np.full(a_matrix.shape[0], -1, dtype=np.int64)
    where[np.asarray(selected, dtype=np.int64)] = np.arange(len(selected))
    keep = where[r] >= 0
    rows = row_offset + where[r[keep]]
    cols, ptrs = c[keep], ptr[keep]
    o = _csc_order(rows, cols)
    return rows[o], cols[o], ptrs[o]


def build_derivative_plan(p_upper: sp.csc_matrix, a_matrix: sp.csc_matrix, l, u) -> OSQPDerivativePlan | None:
    """solver.py:413-571; None without bounds (as the reference)."""
    if l is None or u is None:
        return None
    n, m = p_upper.shape[0], a_matrix.shape[0]
    l = np.asarray(l, dtype=float)
    u = np.asarray(u, dtype=float)
    infval = OSQP_INFTY * OSQP_MIN_SCALING
    ineq = l < u
    lower = np.flatnonzero(ineq & (l > -infval)).astype(np.int32)
    upper = np.flatnonzero(ineq & (u < infval)).astype(np.int32)
    eq = np.flatnonzero(~ineq).astype(np.int32)
    nl, nu, ne = lower.size, upper.size, eq.size
    ni = nl + nu
    half = n + ni + ne
    dim = 2 * half

    p_rows_u, p_cols_u, _ = _entries(p_upper)
    pf_rows, pf_cols, pf_map = full_symmetric_pattern(p_upper)

    lr, lc, lp = selected_rows_pattern(a_matrix, lower, 0)
    ur, uc, up = selected_rows_pattern(a_matrix, upper, nl)
    g_rows = np.concatenate([lr, ur])
    g_cols = np.concatenate([lc, uc])
    g_map = np.concatenate([lp, up])
    g_sign = np.concatenate([np.full(lr.size, -1.0), np.full(ur.size, 1.0)])
    o = _csc_order(g_rows, g_cols)  # the two halves interleave by column
    g_rows, g_cols, g_map, g_sign = g_rows[o], g_cols[o], g_map[o], g_sign[o]
    e_rows, e_cols, e_map = selected_rows_pattern(a_matrix, eq, 0)

    # the blocks of the upper triangle, each as (rows, cols); they never overlap
    ar = np.arange(half, dtype=np.int64)
    ai = np.arange(ni, dtype=np.int64)
    blocks = {
        "diag_first": (ar, ar),
        "p": (pf_rows.astype(np.int64), half + pf_cols.astype(np.int64)),
        "g": (n + g_rows, half + g_cols),
        "aeq": (n + ni + e_rows, half + e_cols),
        "glambda": (g_cols, half + n + g_rows),
        "slack": (n + ai, half + n + ai),
        "aeq_t": (e_cols, half + n + ni + e_rows),
        "diag_second": (half + ar, half + ar),
    }
    all_rows = np.concatenate([b[0] for b in blocks.values()])
    all_cols = np.concatenate([b[1] for b in blocks.values()])
    order = _csc_order(all_rows, all_cols)
    pos_of = np.empty(order.size, dtype=np.int64)
    pos_of[order] = np.arange(order.size)
    indptr = np.zeros(dim + 1, dtype=np.int64)
    np.add.at(indptr, all_cols + 1, 1)
    indptr = np.cumsum(indptr)
    pos, start = {}, 0
    for name, (br, _) in blocks.items():
        pos[name] = pos_of[start : start + br.size].astype(np.int32)
        start += br.size

    data = np.zeros(order.size)
    data[pos["diag_first"]] = 1.0 + ADJOINT_EPS
    data[pos["diag_second"]] = -ADJOINT_EPS
    data[pos["p"]] = np.asarray(p_upper.data, dtype=float)[pf_map]
    data[pos["g"]] = np.asarray(a_matrix.data, dtype=float)[g_map] * g_sign
    data[pos["aeq"]] = np.asarray(a_matrix.data, dtype=float)[e_map]
    data[pos["glambda"]] = 0.0
    data[pos["slack"]] = -1.0
    data[pos["aeq_t"]] = np.asarray(a_matrix.data, dtype=float)[e_map]
    adjoint_upper = sp.csc_matrix((data, all_rows[order].astype(np.int32), indptr.astype(np.int32)), shape=(dim, dim))

    return OSQPDerivativePlan(
        n=n, m=m, n_ineq_l=nl, n_ineq_u=nu, n_eq=ne, adjoint_dim=dim, adjoint_upper=adjoint_upper,
        qdldl_plan=build_qdldl_plan(adjoint_upper, upper=True),
        lower_indices=lower, upper_indices=upper, eq_indices=eq,
        p_upper_rows=p_rows_u.astype(np.int32), p_upper_cols=p_cols_u.astype(np.int32),
        p_full_rows=pf_rows, p_full_cols=pf_cols, p_full_value_map=pf_map,
        g_rows=g_rows.astype(np.int32), g_cols=g_cols.astype(np.int32), g_a_value_map=g_map.astype(np.int32),
        g_sign=g_sign.astype(np.float64),
        aeq_rows=e_rows.astype(np.int32), aeq_cols=e_cols.astype(np.int32), aeq_a_value_map=e_map.astype(np.int32),
        diag_first_pos=pos["diag_first"], diag_second_pos=pos["diag_second"], p_block_pos=pos["p"],
        g_block_pos=pos["g"], aeq_block_pos=pos["aeq"], glambda_block_pos=pos["glambda"],
        slack_diag_pos=pos["slack"], aeq_t_block_pos=pos["aeq_t"], eps=ADJOINT_EPS,
    )
