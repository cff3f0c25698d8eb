"""Batched filter line search on the GPU (mirror of ``warpmpc.jax_sqp.line_search``).

Same names, fields, defaults and argument meaning as
``warpmpc/jax_sqp/line_search.py``; the arrays are ``torch`` CUDA tensors
(NumPy arrays are copied to the current CUDA device) and the work runs in the
library's kernels (``wmpc_constraint_violation``, ``wmpc_filter_line_search``,
``wmpc_sqp_line_search_step``).  Float32 throughout, as the reference's
default SQP dtype.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from .. import native

LINE_SEARCH_MAX_ITER = 0
LINE_SEARCH_CONSTRAINT = 1
LINE_SEARCH_COST = 2
LINE_SEARCH_COST_OR_CONSTRAINT = 3


@dataclass(frozen=True)
class FilterLineSearchSettings:
    """Parameters of the fixed-candidate filter line search (line_search.py:18-29)."""

    line_search_g_max: float = 1e-1
    line_search_g_min: float = 1e-3
    line_search_gamma_c: float = 1e-3
    line_search_armijo_factor: float = 1e-4
    line_search_step_decay: float = 0.5
    line_search_step_min: float = 0.1
    line_search_constraint_scale: float = 0.1
    line_search_cost_accept_uses_trial_cost: bool = True


class FilterLineSearchResult(NamedTuple):
    """Selected step and diagnostics per batch element (line_search.py:32-42)."""

    step_length: object
    cost: object
    constraint_violation: object
    reason: object
    accepted: object
    candidate_costs: object
    candidate_constraint_violations: object
    candidate_acceptance: object


class LineSearchStepResult(NamedTuple):
    """The line-search SQP step after the QP solve (sparse_mpc.py:1047-1052),
    without the QP solve record."""

    z_next: object
    line_search: FilterLineSearchResult
    is_finite: object
    baseline_constraint_violation: object


def make_step_lengths(settings: FilterLineSearchSettings) -> np.ndarray:
    """The static step ladder 1, decay, decay^2, ... >= step_min (line_search.py:45-59)."""
    if not (0.0 < settings.line_search_step_decay < 1.0):
        raise ValueError("line_search_step_decay must be in (0, 1)")
    if settings.line_search_step_min <= 0.0:
        raise ValueError("line_search_step_min must be positive")
    steps: list[float] = []
    step = 1.0
    tolerance = max(1e-12, 1e-12 * settings.line_search_step_min)
    while step + tolerance >= settings.line_search_step_min:
        steps.append(step)
        step *= settings.line_search_step_decay
    if not steps:
        steps.append(1.0)
    return np.asarray(steps, dtype=np.float64)


def _native_settings(settings: FilterLineSearchSettings) -> native.LineSearchSettings:
    return native.LineSearchSettings(
        float(settings.line_search_g_max), float(settings.line_search_g_min), float(settings.line_search_gamma_c),
        float(settings.line_search_armijo_factor), float(settings.line_search_constraint_scale),
        1 if settings.line_search_cost_accept_uses_trial_cost else 0)


def _device(*arrays):
    import torch

    for a in arrays:
        if isinstance(a, torch.Tensor) and a.is_cuda:
            return a.device
    native.require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def _f32(a, device, ndim: int):
    """float32, contiguous, on `device`, with exactly `ndim` dimensions (1-D rows become one-row batches)."""
    import torch

    t = a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))
    t = t.to(device=device, dtype=torch.float32)
    if ndim == 2 and t.dim() == 1:
        t = t[None, :]
    if t.dim() != ndim:
        raise ValueError(f"expected a {ndim}-D array, got shape {tuple(t.shape)}")
    return t.contiguous()


def constraint_violation(lower, g, upper, scale: float):
    """Scaled bound violation ``sqrt(||max(l-g,0)||^2 + ||min(u-g,0)||^2)`` per row (line_search.py:62-69)."""
    import torch

    dev = _device(lower, g, upper)
    g_t = _f32(g, dev, 2)
    lo, up = _f32(lower, dev, 2), _f32(upper, dev, 2)
    if lo.shape != g_t.shape or up.shape != g_t.shape:
        raise ValueError("lower, g and upper must have the same shape")
    batch, m = g_t.shape
    out = torch.empty(batch, dtype=torch.float32, device=dev)
    native.check(native.lib().wmpc_constraint_violation(
        lo.data_ptr(), g_t.data_ptr(), up.data_ptr(), batch, m, float(scale), out.data_ptr(),
        native.current_stream_handle(dev)))
    return out


def filter_line_search_from_evaluations(
    *,
    settings: FilterLineSearchSettings,
    step_lengths,
    baseline_cost,
    baseline_constraint_violation,
    armijo_descent_metric,
    candidate_costs,
    candidate_constraint_violations,
) -> FilterLineSearchResult:
    """Select the first accepted step from precomputed candidate evaluations
    (line_search.py:72-169); candidate arrays have shape ``(n_steps, batch)``."""
    import torch

    dev = _device(step_lengths, baseline_cost, candidate_costs, candidate_constraint_violations)
    steps = _f32(step_lengths, dev, 1)
    cc = _f32(candidate_costs, dev, 2)
    cv = _f32(candidate_constraint_violations, dev, 2)
    n_cand, batch = cc.shape
    if cv.shape != cc.shape:
        raise ValueError("candidate costs and violations must have the same shape")
    bc = _f32(baseline_cost, dev, 1)
    bv = _f32(baseline_constraint_violation, dev, 1)
    am = _f32(armijo_descent_metric, dev, 1)
    if bc.shape[0] != batch or bv.shape[0] != batch or am.shape[0] != batch:
        raise ValueError("baseline arrays must have one entry per batch element")
    step = torch.empty(batch, dtype=torch.float32, device=dev)
    cost = torch.empty_like(step)
    viol = torch.empty_like(step)
    reason = torch.empty(batch, dtype=torch.int32, device=dev)
    accepted = torch.empty(batch, dtype=torch.bool, device=dev)
    acceptance = torch.empty((n_cand, batch), dtype=torch.bool, device=dev)
    s = _native_settings(settings)
    native.check(native.lib().wmpc_filter_line_search(
        ctypes.byref(s), steps.data_ptr(), steps.shape[0], bc.data_ptr(), bv.data_ptr(), am.data_ptr(),
        cc.data_ptr(), cv.data_ptr(), n_cand, batch, step.data_ptr(), cost.data_ptr(), viol.data_ptr(),
        reason.data_ptr(), accepted.data_ptr(), acceptance.data_ptr(), native.current_stream_handle(dev)))
    return FilterLineSearchResult(step, cost, viol, reason, accepted, cc, cv, acceptance)


def line_search_step(
    *,
    settings: FilterLineSearchSettings,
    step_lengths,
    z,
    direction,
    q,
    constraint_l,
    g,
    constraint_u,
    baseline_cost,
    candidate_costs,
    candidate_constraint_violations,
) -> LineSearchStepResult:
    """The SQP line-search step around the filter selection, one kernel launch
    (sparse_mpc.py:1013-1052): the baseline violation of the linearization's
    ``(constraint_l, g, constraint_u)``, the Armijo metric ``sum(q * direction)``,
    the selection over the candidates' evaluations (the NLP's cost and
    constraint violation at ``z + step_k * direction``, shape ``(n_steps,
    batch)``), ``z_next = z + step * direction`` and ``is_finite``."""
    import torch

    dev = _device(z, direction, candidate_costs)
    z_t, d_t, q_t = _f32(z, dev, 2), _f32(direction, dev, 2), _f32(q, dev, 2)
    batch, n = z_t.shape
    if d_t.shape != z_t.shape or q_t.shape != z_t.shape:
        raise ValueError("z, direction and q must have the same shape")
    cl, g_t, cu = _f32(constraint_l, dev, 2), _f32(g, dev, 2), _f32(constraint_u, dev, 2)
    if cl.shape != g_t.shape or cu.shape != g_t.shape or g_t.shape[0] != batch:
        raise ValueError("constraint_l, g and constraint_u must be (batch, m)")
    m = g_t.shape[1]
    steps = _f32(step_lengths, dev, 1)
    cc = _f32(candidate_costs, dev, 2)
    cv = _f32(candidate_constraint_violations, dev, 2)
    if cv.shape != cc.shape or cc.shape[1] != batch:
        raise ValueError("candidate arrays must be (n_steps, batch)")
    bc = _f32(baseline_cost, dev, 1)
    if bc.shape[0] != batch:
        raise ValueError("baseline_cost must have one entry per batch element")
    z_next = torch.empty_like(z_t)
    step = torch.empty(batch, dtype=torch.float32, device=dev)
    cost, viol, bviol = torch.empty_like(step), torch.empty_like(step), torch.empty_like(step)
    reason = torch.empty(batch, dtype=torch.int32, device=dev)
    accepted = torch.empty(batch, dtype=torch.bool, device=dev)
    finite = torch.empty(batch, dtype=torch.bool, device=dev)
    acceptance = torch.empty(cc.shape, dtype=torch.bool, device=dev)
    data = native.SqpStepBatch(
        batch, n, m, steps.shape[0], cc.shape[0], steps.data_ptr(), z_t.data_ptr(), d_t.data_ptr(), q_t.data_ptr(),
        cl.data_ptr(), g_t.data_ptr(), cu.data_ptr(), bc.data_ptr(), cc.data_ptr(), cv.data_ptr(), z_next.data_ptr(),
        step.data_ptr(), cost.data_ptr(), viol.data_ptr(), bviol.data_ptr(), reason.data_ptr(), accepted.data_ptr(),
        finite.data_ptr(), acceptance.data_ptr())
    s = _native_settings(settings)
    native.check(native.lib().wmpc_sqp_line_search_step(ctypes.byref(s), ctypes.byref(data),
                                                        native.current_stream_handle(dev)))
    ls = FilterLineSearchResult(step, cost, viol, reason, accepted, cc, cv, acceptance)
    return LineSearchStepResult(z_next, ls, finite, bviol)
