"""Reverse-mode derivatives of the batched QP solution (torch autograd).

Mirror of the reference's derivative API (``warpmpc/jax_osqp/solver.py``):
``adjoint_derivative_compute`` / ``_get_vec`` / ``_get_mat`` (1046-1192) and
the ``jax.custom_vjp`` wrappers ``solve_primal``, ``solve_xy``, ``solve`` and
``solve_warm_start`` (1238-1472), as ``torch.autograd.Function`` over the C
ABI entry point ``wmpc_osqp_adjoint``.

The backward pass does not factor anything: it solves the active-set adjoint
system on the LDL^T factor the forward solve left in its workspace (see
``wmpc_osqp_adjoint`` in include/warpmpc_b200.h), and assembles the
gradients with the reference's formulas.  Warm-start cotangents are zero, as
in the reference (solver.py:1463-1465); ``z``, residual and objective
cotangents other than ``obj`` are ignored, as in the reference.
"""

from __future__ import annotations

import numpy as np

from .types import FixedOSQPPlan


def _p_matvec(plan: FixedOSQPPlan, p, x):
    import torch

    dev = x.device
    rows = torch.as_tensor(plan.p_full_rows, dtype=torch.long, device=dev)
    cols = torch.as_tensor(plan.p_full_cols, dtype=torch.long, device=dev)
    vmap = torch.as_tensor(plan.p_full_value_map, dtype=torch.long, device=dev)
    upd = p[:, vmap] * x[:, cols]
    out = torch.zeros((x.shape[0], plan.n), dtype=x.dtype, device=dev)
    return out.index_add_(1, rows, upd)


def _match_broadcast(grad, ref):
    if ref.shape[0] == 1 and grad.shape[0] != 1:
        return grad.sum(dim=0, keepdim=True)
    return grad


def _objective_terms(plan, p, q, x, gobj):
    """dx and direct dP/dq contributions of the objective cotangent (solver.py:1336-1355)."""
    import torch

    px = _p_matvec(plan, p.expand(x.shape[0], -1) if p.shape[0] == 1 else p, x)
    dx = gobj[:, None] * (px + q)
    rows = torch.as_tensor(plan.p_upper.indices, dtype=torch.long, device=x.device)
    cols = torch.as_tensor(np.repeat(np.arange(plan.n), np.diff(plan.p_upper.indptr)), dtype=torch.long, device=x.device)
    scale = torch.where(rows == cols, 0.5, 1.0).to(x.dtype)
    dp = gobj[:, None] * scale[None, :] * (x[:, rows] * x[:, cols])
    dq = gobj[:, None] * x
    return dx, dp, dq


def make_derivative_callables(plan: FixedOSQPPlan, engine, adjoint_iters: int | None = None) -> dict:
    import torch

    iters = plan.settings.max_iter if adjoint_iters is None else int(adjoint_iters)

    class _Solve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, warm, p, a, q, l, u):
            x, z, y, prim, dual, obj = engine.solve(p, a, q, l, u, warm=warm, keep_factor=True)
            ctx.ws = engine.last_workspace
            ctx.save_for_backward(p, a, q, l, u, x, z, y)
            ctx.mark_non_differentiable(prim, dual)
            return x, z, y, prim, dual, obj

        @staticmethod
        def backward(ctx, gx, gz, gy, gprim, gdual, gobj):
            p, a, q, l, u, x, z, y = ctx.saved_tensors
            batch = x.shape[0]
            dx = gx if gx is not None else torch.zeros_like(x)
            extra_dp = extra_dq = None
            if gobj is not None and bool(torch.any(gobj != 0)):
                qb = q.expand(batch, -1) if q.shape[0] == 1 else q
                odx, extra_dp, extra_dq = _objective_terms(plan, p, qb, x, gobj)
                dx = dx + odx
            dq, dl, du, dp, da = engine.adjoint(ctx.ws, p, a, l, u, x, z, y, dx.contiguous(),
                                                None if gy is None else gy.contiguous(), max_iter=iters)
            if extra_dp is not None:
                dp = dp + extra_dp
                dq = dq + extra_dq
            return (None, _match_broadcast(dp, p), _match_broadcast(da, a), _match_broadcast(dq, q),
                    _match_broadcast(dl, l), _match_broadcast(du, u))

    def _prep(*tensors):
        out = []
        for t in tensors:
            if not isinstance(t, torch.Tensor):
                t = torch.as_tensor(np.asarray(t, dtype=np.float32))
            t = t.to(engine.device, torch.float32)
            out.append(t[None, :] if t.dim() == 1 else t)
        return out

    def solve(p_values, a_values, q, l, u):
        p, a, qq, ll, uu = _prep(p_values, a_values, q, l, u)
        return _Solve.apply(None, p, a, qq, ll, uu)

    def solve_warm_start(p_values, a_values, q, l, u, warm_start_x, warm_start_z, warm_start_y):
        p, a, qq, ll, uu = _prep(p_values, a_values, q, l, u)
        warm = tuple(t.detach() for t in _prep(warm_start_x, warm_start_z, warm_start_y))
        return _Solve.apply(warm, p, a, qq, ll, uu)

    def solve_primal(p_values, a_values, q, l, u):
        return solve(p_values, a_values, q, l, u)[0]

    def solve_xy(p_values, a_values, q, l, u):
        out = solve(p_values, a_values, q, l, u)
        return out[0], out[2]

    def adjoint_derivative_compute(p_values, a_values, l, u, x, y, dx=None, dy=None, z=None):
        """Gradients for cotangents (dx, dy) at a solution (x, y) (solver.py:1202-1220).

        Factors the KKT matrix once (a zero-iteration solve keeps the factor),
        then runs the adjoint.  ``z`` (the ADMM's projected constraint values)
        fixes the active set; by default it is taken from the sign of ``y``.
        """
        p, a, ll, uu, xx, yy = _prep(p_values, a_values, l, u, x, y)
        batch = xx.shape[0]
        ll = ll.expand(batch, -1).contiguous() if ll.shape[0] == 1 else ll
        uu = uu.expand(batch, -1).contiguous() if uu.shape[0] == 1 else uu
        if z is None:
            zz = torch.where(yy > 0, uu, torch.where(yy < 0, ll, 0.5 * (ll.clamp(min=-1e29) + uu.clamp(max=1e29))))
            zz = torch.where(ll == uu, ll, zz)
        else:
            (zz,) = _prep(z)
        dxx = torch.zeros_like(xx) if dx is None else _prep(dx)[0]
        dyy = None if dy is None else _prep(dy)[0]
        zeros_q = torch.zeros((batch, plan.n), dtype=torch.float32, device=engine.device)
        engine.solve(p, a, zeros_q, ll, uu, keep_factor=True, max_iter=0, check_termination=0)
        ws = engine.last_workspace
        return engine.adjoint(ws, p, a, ll, uu, xx, zz, yy, dxx, dyy, max_iter=iters)

    def adjoint_derivative_get_vec(state):
        dq, dl, du, _, _ = state
        return dq, dl, du

    def adjoint_derivative_get_mat(x, y, state):
        _, _, _, dp, da = state
        return dp, da

    return {
        "solve": solve,
        "solve_warm_start": solve_warm_start,
        "solve_primal": solve_primal,
        "solve_xy": solve_xy,
        "adjoint_derivative_compute": adjoint_derivative_compute,
        "adjoint_derivative_get_vec": adjoint_derivative_get_vec,
        "adjoint_derivative_get_mat": adjoint_derivative_get_mat,
    }
