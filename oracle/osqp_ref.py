"""CPU restatement of the reference's batched fixed-iteration OSQP solve.

TEST INFRASTRUCTURE ONLY (oracle).  Used by ``tests/``, the smoke check and
the CPU-baseline leg of ``bench.py``; never by the product path.

Restates ``warpmpc/jax_osqp/solver.py``:

* ``assemble_kkt_values`` 764-776 (base KKT values with per-instance
  ``P * p_scale + sigma`` and ``A * a_scale`` scattered in);
* ``a_matvec``/``at_matvec``/``p_matvec`` 778-797 (scatter-adds in entry
  order, as ``np.add.at`` does);
* ``_iterate`` 806-820 (one ADMM iteration with over-relaxation);
* ``_solve_with_factor_from_state`` 822-872 (input scaling, ``max_iter``
  iterations, unscaling, residuals and objective);
* ``solve``/``solve_warm_start``/``factor``/``solve_with_factor`` 799-982.

All arrays are batch-major ``(B, .)``; P/A value batches of one broadcast.
Float32 inputs give the reference's float32 path, float64 the truth run.
"""

from __future__ import annotations

import numpy as np

from . import qdldl_ref


def _c(plan, name, dt):
    return np.asarray(getattr(plan, name), dtype=dt)


def assemble_kkt_values(plan, p_values, a_values):
    dt = np.asarray(p_values).dtype
    p_values = np.atleast_2d(np.asarray(p_values, dtype=dt))
    a_values = np.atleast_2d(np.asarray(a_values, dtype=dt))
    batch = max(p_values.shape[0], a_values.shape[0])
    values = np.broadcast_to(np.asarray(plan.kkt_upper.data, dtype=dt), (batch, plan.nnz_kkt)).copy()
    p_upd = p_values * _c(plan, "p_scale", dt)[None, :] + _c(plan, "p_diag_sigma", dt)[None, :]
    a_upd = a_values * _c(plan, "a_scale", dt)[None, :]
    values[:, plan.p_to_kkt] = np.broadcast_to(p_upd, (batch, plan.nnz_p))
    values[:, plan.a_to_kkt] = np.broadcast_to(a_upd, (batch, plan.nnz_a))
    return values


def factor(plan, p_values, a_values):
    """KKT values -> (lx, dinv) in the symbolic-major layout."""
    kkt = assemble_kkt_values(plan, p_values, a_values)
    lx, _, dinv = qdldl_ref.factor(plan.qdldl_plan, kkt.T)
    return lx, dinv


def a_matvec(plan, a_values, x):
    dt = x.dtype
    a_values = np.atleast_2d(np.asarray(a_values, dtype=dt))
    upd = a_values * x[:, plan.a_cols]
    out = np.zeros((x.shape[0], plan.m), dtype=dt)
    for e, row in enumerate(plan.a_rows.tolist()):
        out[:, row] = out[:, row] + upd[:, e]
    return out


def at_matvec(plan, a_values, y):
    dt = y.dtype
    a_values = np.atleast_2d(np.asarray(a_values, dtype=dt))
    upd = a_values * y[:, plan.a_rows]
    out = np.zeros((y.shape[0], plan.n), dtype=dt)
    for e, col in enumerate(plan.a_cols.tolist()):
        out[:, col] = out[:, col] + upd[:, e]
    return out


def p_matvec(plan, p_values, x):
    dt = x.dtype
    p_values = np.atleast_2d(np.asarray(p_values, dtype=dt))
    upd = p_values[:, plan.p_full_value_map] * x[:, plan.p_full_cols]
    out = np.zeros((x.shape[0], plan.n), dtype=dt)
    for e, row in enumerate(plan.p_full_rows.tolist()):
        out[:, row] = out[:, row] + upd[:, e]
    return out


def iterate(plan, state, q, l, u, lx, dinv, dt):
    """One ADMM iteration (solver.py:806-820) in the scaled space."""
    x, z, y = state
    n = plan.n
    sigma = dt.type(plan.settings.sigma)
    alpha = dt.type(plan.settings.alpha)
    rho = _c(plan, "rho_vec", dt)[None, :]
    rho_inv = _c(plan, "rho_inv_vec", dt)[None, :]
    rhs_x = sigma * x - q
    rhs_z = z - rho_inv * y
    rhs = np.concatenate([rhs_x, rhs_z], axis=1)
    sol = qdldl_ref.solve(plan.qdldl_plan, lx, dinv, rhs.T).T
    xt = sol[:, :n]
    zt = rhs_z + rho_inv * sol[:, n:]
    one_minus = dt.type(1.0) - alpha
    x_next = alpha * xt + one_minus * x
    z_rel = alpha * zt + one_minus * z
    z_next = np.minimum(np.maximum(z_rel + rho_inv * y, l), u)
    y_next = y + rho * (z_rel - z_next)
    return x_next, z_next, y_next


def solve_with_factor_from_state(plan, lx, dinv, p_values, a_values, q, l, u, x0, z0, y0, max_iter=None, return_history=False):
    dt = np.asarray(q).dtype
    q = np.atleast_2d(np.asarray(q, dtype=dt))
    l = np.atleast_2d(np.asarray(l, dtype=dt))
    u = np.atleast_2d(np.asarray(u, dtype=dt))
    q_s = q * _c(plan, "q_scale", dt)[None, :]
    l_s = l * _c(plan, "scaling_e", dt)[None, :]
    u_s = u * _c(plan, "scaling_e", dt)[None, :]
    x = np.asarray(x0, dtype=dt) * _c(plan, "scaling_dinv", dt)[None, :]
    z = np.asarray(z0, dtype=dt) * _c(plan, "scaling_e", dt)[None, :]
    y = np.asarray(y0, dtype=dt) * _c(plan, "y_scale", dt)[None, :]
    iters = plan.settings.max_iter if max_iter is None else max_iter
    state = (x, z, y)
    history = []
    for _ in range(iters):
        state = iterate(plan, state, q_s, l_s, u_s, lx, dinv, dt)
        if return_history:
            history.append(state)
    x, z, y = state
    x = x * _c(plan, "scaling_d", dt)[None, :]
    z = z * _c(plan, "scaling_einv", dt)[None, :]
    y = y * _c(plan, "y_unscale", dt)[None, :]
    ax = a_matvec(plan, a_values, x)
    px = p_matvec(plan, p_values, x)
    aty = at_matvec(plan, a_values, y)
    prim = np.max(np.abs(ax - z), axis=1)
    dual = np.max(np.abs(px + q + aty), axis=1)
    obj = dt.type(0.5) * np.sum(x * px, axis=1) + np.sum(q * x, axis=1)
    out = (x, z, y, prim, dual, obj)
    if return_history:
        return out, history
    return out


def solve(plan, p_values, a_values, q, l, u, max_iter=None):
    q = np.atleast_2d(q)
    dt = q.dtype
    lx, dinv = factor(plan, np.asarray(p_values, dtype=dt), np.asarray(a_values, dtype=dt))
    b = q.shape[0]
    zeros_n = np.zeros((b, plan.n), dtype=dt)
    zeros_m = np.zeros((b, plan.m), dtype=dt)
    return solve_with_factor_from_state(plan, lx, dinv, p_values, a_values, q, l, u, zeros_n, zeros_m, zeros_m, max_iter)


def solve_warm_start(plan, p_values, a_values, q, l, u, wx, wz, wy, max_iter=None):
    q = np.atleast_2d(q)
    dt = q.dtype
    lx, dinv = factor(plan, np.asarray(p_values, dtype=dt), np.asarray(a_values, dtype=dt))
    return solve_with_factor_from_state(plan, lx, dinv, p_values, a_values, q, l, u, wx, wz, wy, max_iter)


# ---------------------------------------------------------------------------
# rho adaptation (per instance).  The reference has none (solver.py:587-588
# rejects adaptive_rho); this restates the CUDA path's rule, OSQP's residual
# balancing (Stellato et al. 2020, sec. 5.2) on the scaled iterate, in the
# same float32 operation order: every `interval` iterations (not after the
# last) each instance estimates
#   rho' = clamp(rho sqrt(r_p / (r_d + 1e-10)), 1e-6, 1e6),
#   r_p = |A x - z| / (max(|A x|, |z|) + 1e-10),
#   r_d = |P x + q + A^T y| / (max(|P x|, |A^T y|, |q|) + 1e-10)   (inf-norms),
# takes it when rho' > tol rho or rho' < rho / tol, sets its rho vector by
# the plan's row classes (loose 1e-6, equality 1e3 rho', others rho'),
# 1/rho per row, and refactors its KKT matrix.
# ---------------------------------------------------------------------------


def _iterate_rho(plan, state, q, l, u, lx, dinv, dt, rho, rho_inv):
    """iterate() with per-instance rho vectors rho, rho_inv [B, m]; one factor per instance."""
    x, z, y = state
    n = plan.n
    sigma = dt.type(plan.settings.sigma)
    alpha = dt.type(plan.settings.alpha)
    rhs_x = sigma * x - q
    rhs_z = z - rho_inv * y
    rhs = np.concatenate([rhs_x, rhs_z], axis=1)
    sol = qdldl_ref.solve(plan.qdldl_plan, lx, dinv, rhs.T).T
    xt = sol[:, :n]
    zt = rhs_z + rho_inv * sol[:, n:]
    one_minus = dt.type(1.0) - alpha
    x_next = alpha * xt + one_minus * x
    z_rel = alpha * zt + one_minus * z
    z_next = np.minimum(np.maximum(z_rel + rho_inv * y, l), u)
    y_next = y + rho * (z_rel - z_next)
    return x_next, z_next, y_next


def _factor_rho(plan, p_values, a_values, rho_inv, dt, batch):
    kkt = np.broadcast_to(assemble_kkt_values(plan, p_values, a_values), (batch, plan.nnz_kkt)).copy()
    kkt[:, plan.rho_to_kkt] = -rho_inv
    lx, _, dinv = qdldl_ref.factor(plan.qdldl_plan, kkt.T)
    return lx, dinv


def rho_estimate(plan, p_values, a_values, x, z, y, q_s, rho_b, tol):
    """(take [B] bool, estimate [B]) of the rule above on the scaled iterate."""
    dt = x.dtype
    f = dt.type
    a_s = np.atleast_2d(np.asarray(a_values, dtype=dt)) * _c(plan, "a_scale", dt)[None, :]
    p_s = np.atleast_2d(np.asarray(p_values, dtype=dt)) * _c(plan, "p_scale", dt)[None, :]
    ax = a_matvec(plan, a_s, x)
    px = p_matvec(plan, p_s, x)
    aty = at_matvec(plan, a_s, y)
    prim = np.max(np.abs(ax - z), axis=1)
    pn = np.maximum(np.max(np.abs(ax), axis=1), np.max(np.abs(z), axis=1))
    dual = np.max(np.abs(px + q_s + aty), axis=1)
    dn = np.maximum(np.maximum(np.max(np.abs(px), axis=1), np.max(np.abs(aty), axis=1)),
                    np.max(np.abs(q_s), axis=1))
    rp = prim / (pn + f(1e-10))
    rd = dual / (dn + f(1e-10))
    est = rho_b * np.sqrt(rp / (rd + f(1e-10)))
    est = np.minimum(np.maximum(est, f(1e-6)), f(1e6))
    take = (est > rho_b * f(tol)) | (est < rho_b / f(tol))
    return take, est.astype(dt)


def solve_adaptive(plan, p_values, a_values, q, l, u, warm=None, max_iter=None, interval=None, tol=None):
    """solve()/solve_warm_start() with per-instance rho adaptation.
    Returns (x, z, y, prim, dual, obj, rho [B], rho_updates [B])."""
    q = np.atleast_2d(q)
    dt = q.dtype
    f = dt.type
    s = plan.settings
    iters = s.max_iter if max_iter is None else max_iter
    interval = s.adaptive_rho_interval if interval is None else interval
    tol = s.adaptive_rho_tolerance if tol is None else tol
    l = np.atleast_2d(np.asarray(l, dtype=dt))
    u = np.atleast_2d(np.asarray(u, dtype=dt))
    b = max(q.shape[0], l.shape[0], np.atleast_2d(p_values).shape[0], np.atleast_2d(a_values).shape[0])
    rho = np.broadcast_to(_c(plan, "rho_vec", dt)[None, :], (b, plan.m)).copy()
    rho_inv = np.broadcast_to(_c(plan, "rho_inv_vec", dt)[None, :], (b, plan.m)).copy()
    rho_b = np.full(b, f(s.rho), dtype=dt)
    count = np.zeros(b, dtype=np.int32)
    pv, av = np.asarray(p_values, dtype=dt), np.asarray(a_values, dtype=dt)
    lx, dinv = _factor_rho(plan, pv, av, rho_inv, dt, b)
    q_s = np.broadcast_to(q * _c(plan, "q_scale", dt)[None, :], (b, plan.n))
    l_s = l * _c(plan, "scaling_e", dt)[None, :]
    u_s = u * _c(plan, "scaling_e", dt)[None, :]
    if warm is None:
        x = np.zeros((b, plan.n), dt)
        z = np.zeros((b, plan.m), dt)
        y = np.zeros((b, plan.m), dt)
    else:
        x = np.asarray(warm[0], dtype=dt) * _c(plan, "scaling_dinv", dt)[None, :]
        z = np.asarray(warm[1], dtype=dt) * _c(plan, "scaling_e", dt)[None, :]
        y = np.asarray(warm[2], dtype=dt) * _c(plan, "y_scale", dt)[None, :]
    ctype = np.asarray(plan.constr_type)
    for it in range(iters):
        x, z, y = _iterate_rho(plan, (x, z, y), q_s, l_s, u_s, lx, dinv, dt, rho, rho_inv)
        if (it + 1) % interval == 0 and it + 1 < iters:
            take, est = rho_estimate(plan, pv, av, x, z, y, q_s, rho_b, tol)
            if np.any(take):
                rho_b = np.where(take, est, rho_b).astype(dt)
                count += take.astype(np.int32)
                new = np.where(ctype[None, :] < 0, f(1e-6),
                               np.where(ctype[None, :] > 0, f(1e3) * rho_b[:, None], rho_b[:, None])).astype(dt)
                rho = np.where(take[:, None], new, rho)
                rho_inv = np.where(take[:, None], f(1.0) / new, rho_inv)
                lx, dinv = _factor_rho(plan, pv, av, rho_inv, dt, b)
    x = x * _c(plan, "scaling_d", dt)[None, :]
    z = z * _c(plan, "scaling_einv", dt)[None, :]
    y = y * _c(plan, "y_unscale", dt)[None, :]
    ax = a_matvec(plan, a_values, x)
    px = p_matvec(plan, p_values, x)
    aty = at_matvec(plan, a_values, y)
    prim = np.max(np.abs(ax - z), axis=1)
    dual = np.max(np.abs(px + q + aty), axis=1)
    obj = f(0.5) * np.sum(x * px, axis=1) + np.sum(q * x, axis=1)
    return x, z, y, prim, dual, obj, rho_b, count
