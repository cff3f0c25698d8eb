"""The primal-residual recursion the streaming kernel's termination test uses.

The kernel never forms A x: it carries the scaled primal residual
e_k = A x_k - z_k from its start value through the iterations as

    e_{k+1} = (z_relaxed - z_{k+1}) + (1 - alpha) e_k,

which holds because the KKT solve returns x~, z~ with A x~ = z~
(``warpmpc/jax_osqp/solver.py`` 806-820: x_{k+1} = alpha x~ + (1 - alpha) x_k,
z_relaxed = alpha z~ + (1 - alpha) z_k).  These tests replay the oracle's
iterations in float64 and check the recursion against A x_k - z_k at every
iteration, cold and warm started.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import osqp_ref, qdldl_ref
from warpmpc_b200 import problems


def _scaled_a(plan, a_values):
    return np.atleast_2d(a_values) * np.asarray(plan.a_scale, dtype=np.float64)[None, :]


def _replay(plan, b, x0, z0, y0, iters):
    """Oracle iterations in float64; returns (recursion e_k, exact A x_k - z_k) per k."""
    f = np.float64
    p, a = b.p_values.astype(f), b.a_values.astype(f)
    q = np.atleast_2d(b.q).astype(f) * np.asarray(plan.q_scale, f)[None, :]
    l = np.atleast_2d(b.l).astype(f) * np.asarray(plan.scaling_e, f)[None, :]
    u = np.atleast_2d(b.u).astype(f) * np.asarray(plan.scaling_e, f)[None, :]
    lx, dinv = osqp_ref.factor(plan, p, a)
    x = x0.astype(f) * np.asarray(plan.scaling_dinv, f)[None, :]
    z = z0.astype(f) * np.asarray(plan.scaling_e, f)[None, :]
    y = y0.astype(f) * np.asarray(plan.y_scale, f)[None, :]
    a_hat = _scaled_a(plan, a)
    alpha = f(plan.settings.alpha)
    rho_inv = np.asarray(plan.rho_inv_vec, f)[None, :]
    e = osqp_ref.a_matvec(plan, a_hat, x) - z
    out = []
    for _ in range(iters):
        # z_relaxed as the iteration forms it (before projection)
        rhs_z = z - rho_inv * y
        x_n, z_n, y_n = osqp_ref.iterate(plan, (x, z, y), q, l, u, lx, dinv, np.dtype(f))
        rhs = np.concatenate([f(plan.settings.sigma) * x - q, rhs_z], axis=1)
        sol = qdldl_ref.solve(plan.qdldl_plan, lx, dinv, rhs.T).T
        zt = rhs_z + rho_inv * sol[:, plan.n:]
        z_rel = alpha * zt + (1.0 - alpha) * z
        e = (z_rel - z_n) + (1.0 - alpha) * e
        x, z, y = x_n, z_n, y_n
        out.append((e.copy(), osqp_ref.a_matvec(plan, a_hat, x) - z))
    return out


@pytest.mark.parametrize("warm", [False, True])
def test_primal_residual_recursion_matches_ax_minus_z(warm):
    b = problems.make_batch(problems.SMALL, 6, seed=3)
    plan = problems.make_plan(b)
    bs = b.q.shape[0]
    if warm:
        rng = np.random.default_rng(11)
        x0 = rng.standard_normal((bs, plan.n))
        z0 = rng.standard_normal((bs, plan.m))
        y0 = rng.standard_normal((bs, plan.m))
    else:
        x0, z0, y0 = np.zeros((bs, plan.n)), np.zeros((bs, plan.m)), np.zeros((bs, plan.m))
    steps = _replay(plan, b, x0, z0, y0, 30)
    for k, (rec, exact) in enumerate(steps):
        scale = 1.0 + np.max(np.abs(exact))
        assert np.max(np.abs(rec - exact)) <= 1e-9 * scale, f"iteration {k + 1}"


def test_primal_residual_start_value_cold_is_zero():
    b = problems.make_batch(problems.QUADROTOR, 3, seed=1)
    plan = problems.make_plan(b)
    x = np.zeros((3, plan.n))
    z = np.zeros((3, plan.m))
    assert not np.any(osqp_ref.a_matvec(plan, _scaled_a(plan, b.a_values.astype(np.float64)), x) - z)
