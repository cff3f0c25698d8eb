"""CPU restatement of the reference's batched QDLDL factor and solve.

TEST INFRASTRUCTURE ONLY (oracle).  Used by ``tests/``, the smoke check and
the CPU-baseline leg of ``bench.py``; never by the product path.

Restates, vectorised over the batch (symbolic-major ``(rows, batch)`` layout):

* numeric factorization -- ``warpmpc/jax_qdldl/warp_backend.py:41-101``
  (``_qdldl_factor_transpose_kernel``) and ``warpmpc/jax_qdldl/core.py:867-933``
  (``factor_symbolic``): per row ``k``, gather the permuted KKT column, scatter
  it into the work vector ``y``, then for each column ``cidx`` of the row
  program: ``y[rows] += -lx * val`` over the first ``offset`` entries of
  column ``cidx``, ``lval = val * dinv[cidx]``, ``d_k -= val * lval``;
  finally ``dinv[k] = 1 / d_k``;
* triangular solve -- ``warp_backend.py:176-218``
  (``_qdldl_solve_serial_transpose_kernel``): permute, column-oriented forward
  substitution with L, scale by ``dinv``, row-oriented backward substitution
  with L^T, unpermute.

Arithmetic follows the reference's operation order with every product and
sum rounded separately (NumPy does not contract multiply-add), in the dtype of
the inputs: float32 for parity, float64 for truth.
"""

from __future__ import annotations

import numpy as np


def factor(plan, a_values: np.ndarray):
    """``a_values`` ``(nnz_a, B)`` in original upper-CSC order -> ``(lx, d, dinv)``."""

    a_values = np.asarray(a_values)
    dt = a_values.dtype
    n = plan.n
    batch = a_values.shape[1]
    a_perm = a_values[plan.perm_to_orig, :]
    y = np.zeros((n, batch), dtype=dt)
    lx = np.zeros((plan.nnz_l, batch), dtype=dt)
    d = np.zeros((n, batch), dtype=dt)
    dinv = np.zeros((n, batch), dtype=dt)
    one = dt.type(1.0)
    zero = dt.type(0.0)
    lp = plan.lp
    li = plan.li
    for k in range(n):
        d_k = a_perm[plan.diag_pos[k], :].copy()
        m_init = plan.init_mask[k]
        rows = plan.init_rows[k][m_init]
        pos = plan.init_pos[k][m_init]
        for row, ptr in zip(rows.tolist(), pos.tolist()):
            y[row, :] = y[row, :] + a_perm[ptr, :]
        m_proc = plan.process_mask[k]
        cols = plan.process_cols[k][m_proc].tolist()
        dests = plan.process_lidx[k][m_proc].tolist()
        offs = plan.process_offsets[k][m_proc].tolist()
        for cidx, dest, off in zip(cols, dests, offs):
            val = y[cidx, :].copy()
            if off:
                seg = slice(lp[cidx], lp[cidx] + off)
                # rows of one L column are distinct: the scatter has no collisions
                y[li[seg], :] = y[li[seg], :] + (-lx[seg, :]) * val[None, :]
            lval = val * dinv[cidx, :]
            lx[dest, :] = lval
            d_k = d_k - val * lval
        d[k, :] = d_k
        dinv[k, :] = one / d_k
        if cols:
            y[cols, :] = zero
    return lx, d, dinv


def solve(plan, lx: np.ndarray, dinv: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """``rhs`` ``(n, B)`` -> ``x`` with ``x = P^T L^-T D^-1 L^-1 P rhs``.

    ``lx``/``dinv`` with a batch of one are broadcast over ``rhs``'s batch.
    """

    rhs = np.asarray(rhs)
    dt = rhs.dtype
    n = plan.n
    lp = plan.lp
    li = plan.li
    work = rhs[plan.p, :].copy()
    for col in range(n):
        a, b = lp[col], lp[col + 1]
        if b > a:
            val = work[col, :]
            work[li[a:b], :] = work[li[a:b], :] + (-lx[a:b, :]) * val[None, :]
    work = work * dinv
    for col in range(n - 1, -1, -1):
        a, b = lp[col], lp[col + 1]
        corr = np.zeros(work.shape[1], dtype=dt)
        for e in range(a, b):
            corr = corr + lx[e, :] * work[li[e], :]
        work[col, :] = work[col, :] - corr
    return work[plan.pinv, :]


def factor_and_solve(plan, a_values, rhs):
    lx, d, dinv = factor(plan, a_values)
    return solve(plan, lx, dinv, rhs), lx, d


def dense_kkt(plan, a_values_column: np.ndarray) -> np.ndarray:
    """Dense symmetric matrix of one instance (float64), for residual checks."""
    n = plan.n
    out = np.zeros((n, n), dtype=np.float64)
    cols = np.repeat(np.arange(n), np.diff(plan.a_indptr))
    out[plan.a_indices, cols] = a_values_column
    out = out + np.triu(out, 1).T
    return out
