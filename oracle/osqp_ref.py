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
