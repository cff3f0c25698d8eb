"""CPU restatement of the reference's filter line search and line-search step.

TEST INFRASTRUCTURE ONLY (oracle).  Used by ``tests/`` and the CPU leg of
``bench.py``; never by the product path.

Restates ``warpmpc/jax_sqp/line_search.py``:

* ``make_step_lengths`` 45-59 (the step ladder, float64);
* ``constraint_violation`` 62-69 (scaled bound violation);
* ``filter_line_search_from_evaluations`` 72-169 (per-candidate branch and
  acceptance, first accepted candidate, fallback to the last step);

and the step around it in ``warpmpc/jax_sqp/sparse_mpc.py`` 1013-1052
(baseline violation, Armijo metric ``sum(q * d)``, ``z + step * d``,
``is_finite``).  Arrays follow the reference's shapes: candidates
``(n_steps, batch)``, rows ``(batch, .)``; float32 inputs give the
reference's float32 path element by element.
"""

from __future__ import annotations

import numpy as np

MAX_ITER, CONSTRAINT, COST, COST_OR_CONSTRAINT = 0, 1, 2, 3


def make_step_lengths(step_decay: float, step_min: float) -> np.ndarray:
    """line_search.py:45-59."""
    if not (0.0 < step_decay < 1.0):
        raise ValueError("line_search_step_decay must be in (0, 1)")
    if step_min <= 0.0:
        raise ValueError("line_search_step_min must be positive")
    steps = []
    step = 1.0
    tol = max(1e-12, 1e-12 * step_min)
    while step + tol >= step_min:
        steps.append(step)
        step *= step_decay
    if not steps:
        steps.append(1.0)
    return np.asarray(steps, dtype=np.float64)


def constraint_violation(lower, g, upper, scale):
    """line_search.py:62-69 (the two squared sums formed separately)."""
    g = np.asarray(g)
    dt = g.dtype
    lo_gap = np.asarray(lower, dt) - g
    up_gap = np.asarray(upper, dt) - g
    a = np.maximum(lo_gap, dt.type(0))
    c = np.minimum(up_gap, dt.type(0))
    vsq = np.sum(a * a, axis=1, dtype=dt) + np.sum(c * c, axis=1, dtype=dt)
    return dt.type(scale) * np.sqrt(vsq)


def filter_line_search(settings: dict, step_lengths, baseline_cost, baseline_violation, armijo_metric,
                       candidate_costs, candidate_violations):
    """line_search.py:72-169.  ``settings`` holds g_max, g_min, gamma_c,
    armijo_factor, cost_accept_uses_trial_cost.  Returns (step, cost,
    violation, reason, accepted, acceptance[n_cand, batch])."""
    cc = np.asarray(candidate_costs)
    dt = cc.dtype
    cv = np.asarray(candidate_violations, dt)
    steps = np.asarray(step_lengths, dt)
    bc = np.asarray(baseline_cost, dt)[None, :]
    bv = np.asarray(baseline_violation, dt)[None, :]
    am = np.asarray(armijo_metric, dt)[None, :]
    g_max, g_min = dt.type(settings["g_max"]), dt.type(settings["g_min"])
    gamma_c, armijo_factor = dt.type(settings["gamma_c"]), dt.type(settings["armijo_factor"])
    one_minus_gamma = dt.type(1.0) - gamma_c
    constraint_reason = cv > g_max
    constraint_accept = cv < one_minus_gamma * bv
    cost_reason = (cv < g_min) & (bv < g_min) & (am < dt.type(0))
    lhs = cc if settings.get("cost_accept_uses_trial_cost", True) else np.broadcast_to(bc, cc.shape)
    cost_accept = lhs < (bc + armijo_factor * am)
    filter_accept = (cc < (bc - gamma_c * bv)) | (cv < one_minus_gamma * bv)
    accepted = np.where(constraint_reason, constraint_accept, np.where(cost_reason, cost_accept, filter_accept))
    reason = np.where(constraint_reason, CONSTRAINT, np.where(cost_reason, COST, COST_OR_CONSTRAINT))
    any_acc = accepted.any(axis=0)
    first = np.argmax(accepted.astype(np.int32), axis=0)
    sel = np.where(any_acc, first, steps.shape[0] - 1)
    b = np.arange(cc.shape[1])
    ci = np.minimum(sel, cc.shape[0] - 1)  # gathers clamp, as the reference's do
    si = np.minimum(sel, steps.shape[0] - 1)
    sel_reason = np.where(any_acc, reason[ci, b], MAX_ITER).astype(np.int32)
    return steps[si], cc[ci, b], cv[ci, b], sel_reason, any_acc, accepted


def line_search_step(settings: dict, step_lengths, z, direction, q, constraint_l, g, constraint_u, baseline_cost,
                     candidate_costs, candidate_violations):
    """sparse_mpc.py:1013-1052 after the QP solve: returns (z_next, is_finite,
    baseline_violation, armijo metric, filter result)."""
    z = np.asarray(z)
    dt = z.dtype
    bviol = constraint_violation(constraint_l, g, constraint_u, settings["constraint_scale"])
    armijo = np.sum(np.asarray(q, dt) * np.asarray(direction, dt), axis=1, dtype=dt)
    res = filter_line_search(settings, step_lengths, baseline_cost, bviol, armijo, candidate_costs,
                             candidate_violations)
    z_next = z + res[0][:, None] * np.asarray(direction, dt)
    return z_next, np.all(np.isfinite(z_next), axis=1), bviol, armijo, res
