"""One SQP step with the filter line search, every stage after the model on the GPU.

Mirror of ``_line_search_step_with_state_jit`` (``warpmpc/jax_sqp/
sparse_mpc.py:997-1053``) and the pieces it calls: the linearization at z
(stage evaluation by the caller's model, assembly by ``wmpc_sqp_assemble``),
the warm-started QP solve (the persistent OSQP kernel of the plan's OSQP
plan), the candidates ``z + step_k d`` of the step ladder (values-only stage
evaluations, assembled rows, bound violation by ``wmpc_constraint_violation``)
and the filter selection with ``z_next`` (``wmpc_sqp_line_search_step``).

The model is a callable ``evaluate(z, params, values_only)`` returning, per
stage, ``(cost, g, lower, upper)`` and, unless ``values_only``, also
``(grad, hess, jac)`` in the stage's pattern order (batch-major float32
tensors) -- the role of the reference's CasADi stage functions.  A step is a
fixed sequence of launches with no host synchronization, so it can be
captured in a CUDA graph and replayed (the reference jit-compiles the same
sequence).
"""

from __future__ import annotations

from typing import Callable, NamedTuple

import numpy as np

from ..jax_osqp import compile_osqp
from .assembly import QPAssembler, SparseMPCPlan, SparseMPCProblem, SQPLinearization
from .line_search import FilterLineSearchResult, FilterLineSearchSettings, line_search_step, make_step_lengths
from .. import native


class SQPSolveResult(NamedTuple):
    """The QP subproblem at one iterate (types.py:28-37)."""

    direction: object
    z: object
    y: object
    prim_res: object
    dual_res: object
    obj_val: object
    linearization: SQPLinearization


class SQPLineSearchStepResult(NamedTuple):
    """One SQP step with the filter line search (types.py:47-53)."""

    z_next: object
    solve: SQPSolveResult
    line_search: FilterLineSearchResult
    is_finite: object


class SparseMPCSQP:
    """Batched SQP steps of one problem on one device."""

    def __init__(self, problem: SparseMPCProblem, plan: SparseMPCPlan, evaluate: Callable, device=None,
                 line_search_settings: FilterLineSearchSettings | None = None, mode: str = "persistent"):
        import torch

        native.require_cuda()
        self.problem, self.plan, self.evaluate = problem, plan, evaluate
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.settings = line_search_settings or FilterLineSearchSettings()
        steps = make_step_lengths(self.settings).astype(np.float32)
        self.step_lengths = torch.as_tensor(steps, device=self.device)
        self._steps_host = [float(s) for s in steps]
        self.assembler = QPAssembler(plan, problem, self.device)
        self.values = QPAssembler(plan, problem, self.device, values_only=True)
        self.qp = compile_osqp(plan.osqp_plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode=mode,
                               device=self.device)
        self._qp_ws = None  # one QP workspace for every solve of a batch size (sized for a kept factorization)

    def linearize(self, z, params) -> SQPLinearization:
        """_linearize_jit (sparse_mpc.py:855-901)."""
        return self.assembler.assemble(self.assembler.pack(self.evaluate(z, params, False)))

    def evaluate_nlp(self, z, params):
        """_evaluate_values (sparse_mpc.py:840-853): (cost, g, lower, upper)."""
        r = self.values.assemble(self.values.pack(self.evaluate(z, params, True)))
        return r.cost, r.g, r.constraint_l, r.constraint_u

    def solve_qp(self, z, params, warm, keep_factor: bool = False) -> SQPSolveResult:
        """_solve_qp_with_state_jit (sparse_mpc.py:954-976): the QP at z, warm-started.
        keep_factor: the QP engine keeps the factorization for an adjoint."""
        import torch

        lin = self.linearize(z, params)
        eng = self.qp.engine
        batch = int(lin.q.shape[0])
        need = eng.workspace_bytes(batch, keep_factor=True)
        if self._qp_ws is None or self._qp_ws.numel() < need:
            self._qp_ws = None
            self._qp_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        x, qz, qy, prim, dual, obj = eng.solve(lin.p_values, lin.a_values, lin.q, lin.l, lin.u, warm=warm,
                                               keep_factor=keep_factor, workspace=self._qp_ws)
        return SQPSolveResult(x, qz, qy, prim, dual, obj, lin)

    def line_search_step(self, z, params, warm, keep_factor: bool = False) -> SQPLineSearchStepResult:
        """_line_search_step_with_state_jit (sparse_mpc.py:997-1053)."""
        import torch

        from .line_search import constraint_violation

        solve = self.solve_qp(z, params, warm, keep_factor)
        d = solve.direction
        costs, viols = [], []
        for step in self._steps_host:
            c, g, lo, up = self.evaluate_nlp(z + step * d, params)
            costs.append(c)
            viols.append(constraint_violation(lo, g, up, self.settings.line_search_constraint_scale))
        base = solve.linearization
        r = line_search_step(settings=self.settings, step_lengths=self.step_lengths, z=z, direction=d, q=base.q,
                             constraint_l=base.constraint_l, g=base.g, constraint_u=base.constraint_u,
                             baseline_cost=base.cost, candidate_costs=torch.stack(costs),
                             candidate_constraint_violations=torch.stack(viols))
        return SQPLineSearchStepResult(r.z_next, solve, r.line_search, r.is_finite)
