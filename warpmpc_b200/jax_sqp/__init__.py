"""SQP outer-loop pieces with a CUDA backend.

Mirror of ``warpmpc.jax_sqp`` for the sparse MPC plan and batched QP
assembly (``warpmpc/jax_sqp/sparse_mpc.py`` 532-691, 855-901), the filter
line search (``warpmpc/jax_sqp/line_search.py``) and the line-search step
that follows the QP solve (``sparse_mpc.py`` 997-1053).
"""

from .assembly import (
    QPAssembler,
    SparseMPCPlan,
    SparseMPCProblem,
    SQPLinearization,
    StageAssembly,
    build_sparse_mpc_plan,
)
from .sqp import SparseMPCSQP, SQPLineSearchStepResult, SQPSolveResult
from .line_search import (
    LINE_SEARCH_CONSTRAINT,
    LINE_SEARCH_COST,
    LINE_SEARCH_COST_OR_CONSTRAINT,
    LINE_SEARCH_MAX_ITER,
    FilterLineSearchResult,
    FilterLineSearchSettings,
    LineSearchStepResult,
    constraint_violation,
    filter_line_search_from_evaluations,
    line_search_step,
    make_step_lengths,
)

__all__ = [
    "QPAssembler",
    "SQPLinearization",
    "SparseMPCPlan",
    "SparseMPCProblem",
    "SparseMPCSQP",
    "SQPLineSearchStepResult",
    "SQPSolveResult",
    "StageAssembly",
    "build_sparse_mpc_plan",
    "FilterLineSearchResult",
    "FilterLineSearchSettings",
    "LINE_SEARCH_CONSTRAINT",
    "LINE_SEARCH_COST",
    "LINE_SEARCH_COST_OR_CONSTRAINT",
    "LINE_SEARCH_MAX_ITER",
    "LineSearchStepResult",
    "constraint_violation",
    "filter_line_search_from_evaluations",
    "line_search_step",
    "make_step_lengths",
]
