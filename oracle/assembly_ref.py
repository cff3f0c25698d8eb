"""CPU restatement of the reference's sparse MPC QP assembly.

TEST INFRASTRUCTURE ONLY (oracle).

Restates the scatter half of ``_linearize_jit``
(``warpmpc/jax_sqp/sparse_mpc.py:855-901``): starting from zeros, every
stage in order adds its gradient into q at ``q_cols``, its Hessian values
into P at ``p_pos`` and its Jacobian values into A at ``a_pos`` (entries in
the stage's order, one float32 addition each); the constraint rows take
``l = lower - g``, ``u = upper - g`` and keep g, lower and upper; the cost is
the stage costs added in stage order.
"""

from __future__ import annotations

import numpy as np


def assemble(plan, problem, stage_values, values_only=False):
    """stage_values: per stage (cost [B], g, lower, upper [B, nc], grad, hess,
    jac [B, k]) float32 arrays (values_only: the first four; the derivative
    outputs stay zero, as _evaluate_values has none, sparse_mpc.py:840-853).
    Returns the nine SQPLinearization arrays."""
    f = np.float32
    b = np.asarray(stage_values[0][0]).shape[0]
    n, m = int(plan.z_offsets[-1]), int(plan.constraint_offsets[-1])
    q = np.zeros((b, n), f)
    pv = np.zeros((b, plan.p_pattern.nnz), f)
    av = np.zeros((b, plan.a_pattern.nnz), f)
    g_all, lo_all, up_all = np.zeros((b, m), f), np.zeros((b, m), f), np.zeros((b, m), f)
    cost = np.zeros(b, f)
    for st, asm, vals in zip(problem.stages, plan.assemblies, stage_values):
        c, g, lo, up = (np.asarray(v, f) for v in vals[:4])
        r0, nc = asm.constraint_offset, st.constraint_dim
        g_all[:, r0 : r0 + nc] = g
        lo_all[:, r0 : r0 + nc] = lo
        up_all[:, r0 : r0 + nc] = up
        cost = cost + c
        if values_only:
            continue
        grad, hess, jac = (np.asarray(v, f) for v in vals[4:7])
        for j, col in enumerate(asm.q_cols):
            q[:, col] = q[:, col] + grad[:, j]
        for j, pos in enumerate(asm.p_pos):
            pv[:, pos] = pv[:, pos] + hess[:, j]
        for j, pos in enumerate(asm.a_pos):
            av[:, pos] = av[:, pos] + jac[:, j]
    return pv, av, q, lo_all - g_all, up_all - g_all, cost, g_all, lo_all, up_all
