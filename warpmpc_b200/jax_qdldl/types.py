"""Plan and compiled-solver records for the fixed-pattern batched LDL^T path.

Field-for-field mirror of the reference records ``QDLDLPlan`` and
``CompiledQDLDL`` (``warpmpc/jax_qdldl/types.py:11-69``) so code written
against the reference reads the same attributes.  Arrays are NumPy on the
host; compiled callables take and return ``torch`` CUDA tensors.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np


@dataclass(frozen=True)
class QDLDLPlan:
    """All pattern-dependent data of one fixed sparsity pattern."""

    n: int
    nnz_a: int
    nnz_l: int
    a_indptr: np.ndarray
    a_indices: np.ndarray
    a_data: np.ndarray
    aperm_indptr: np.ndarray
    aperm_indices: np.ndarray
    perm_to_orig: np.ndarray
    orig_to_perm: np.ndarray
    p: np.ndarray
    pinv: np.ndarray
    etree: np.ndarray
    lnz: np.ndarray
    lp: np.ndarray
    li: np.ndarray
    diag_pos: np.ndarray
    init_rows: np.ndarray
    init_pos: np.ndarray
    init_mask: np.ndarray
    process_cols: np.ndarray
    process_lidx: np.ndarray
    process_offsets: np.ndarray
    process_mask: np.ndarray
    col_rows: np.ndarray
    col_lidx: np.ndarray
    col_mask: np.ndarray

    @property
    def max_init(self) -> int:
        return int(self.init_rows.shape[1])

    @property
    def max_row_nnz(self) -> int:
        return int(self.process_cols.shape[1])

    @property
    def max_col_nnz(self) -> int:
        return int(self.col_rows.shape[1])


@dataclass(frozen=True)
class CompiledQDLDL:
    """Compiled fixed-pattern factor and solve callables.

    ``backend="cuda"``: ``factor(values (nnz_a, B)) -> (lx (nnz_l, B), d (n, B),
    dinv (n, B))``; ``solve(lx, dinv, rhs (n, B)) -> x (n, B)``;
    ``factor_and_solve(values, rhs) -> (x, lx, d)``.  A batch of one in
    ``lx``/``dinv`` is broadcast over the right-hand-side batch.
    """

    plan: QDLDLPlan
    dtype: np.dtype
    factor: Callable
    solve: Callable
    factor_and_solve: Callable
    variant: str = "baseline"
    values_layout: str = "original_batch"
    rhs_layout: str = "batch"
    backend: str = "jax"
    factor_backend: str = "jax"
    solve_backend: str = "jax"
    device_plan: Any = field(default=None, compare=False, repr=False)
