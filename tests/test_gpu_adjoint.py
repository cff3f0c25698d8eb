"""Adjoint (reverse-mode) derivatives on the GPU.

Checked against (1) the exact active-set derivative computed in float64 from
the GPU's own forward solution, (2) central finite differences of float64
oracle solves (the C restatement, converged), and (3) the restated reference
gradient path (looser: the reference's eps-regularized augmented solve is
itself a few percent off the exact derivative on some instances).
"""

import numpy as np
import pytest

from oracle import adjoint_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp

pytestmark = pytest.mark.gpu

ITERS = 1500


def _setup(cls, batch, seed, iters=ITERS):
    b = problems.make_batch(cls, batch, seed=seed)
    plan = problems.make_plan(b, OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": iters}))
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent",
                        derivatives=True, adjoint_iters=iters)
    return b, plan, comp


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-8, np.max(np.abs(b))))


@pytest.mark.parametrize("cls", [problems.SMALL, problems.CARTPOLE], ids=lambda c: c.name)
def test_adjoint_matches_exact_derivative(cuda_device, cls):
    b, plan, comp = _setup(cls, 16, seed=31)
    eng = comp.engine
    x, z, y, prim, dual, obj = eng.solve(_t(b.p_values), _t(b.a_values), _t(b.q), _t(b.l), _t(b.u), keep_factor=True)
    rng = np.random.default_rng(4)
    dx = rng.standard_normal((16, plan.n)).astype(np.float32)
    dy = rng.standard_normal((16, plan.m)).astype(np.float32)
    got = eng.adjoint(eng.last_workspace, _t(b.p_values), _t(b.a_values), _t(b.l), _t(b.u), x, z, y, _t(dx), _t(dy))
    got = [g.cpu().numpy() for g in got]
    X, Z, Y = (v.cpu().numpy().astype(np.float64) for v in (x, z, y))
    worst = 0.0
    for i in range(16):
        ref = adjoint_ref.active_set_adjoint(plan, b.p_values[i].astype(np.float64), b.a_values[i].astype(np.float64),
                                             b.l[i].astype(np.float64), b.u[i].astype(np.float64), X[i], Z[i], Y[i],
                                             dx[i].astype(np.float64), dy[i].astype(np.float64))
        for g, r in zip((got[0][i], got[1][i], got[2][i], got[3][i], got[4][i]), ref):
            worst = max(worst, _rel(g, r))
    assert worst < 2e-3, worst


def test_adjoint_against_finite_differences(cuda_device):
    """d/d(x0, diag Q) of ||u0 - u_target||^2 (cartpole-like class), via torch autograd."""
    import torch

    from oracle.cpu_baseline import CpuOSQP

    cls = problems.CARTPOLE
    b, plan, comp = _setup(cls, 4, seed=41)
    u_target = np.random.default_rng(2).standard_normal((4, cls.nu))
    ui = (cls.horizon + 1) * cls.nx  # first input variable
    p = _t(b.p_values).requires_grad_(True)
    lo = _t(b.l).requires_grad_(True)
    hi = _t(b.u).requires_grad_(True)
    x = comp.solve_primal(p, _t(b.a_values), _t(b.q), lo, hi)
    loss = ((x[:, ui : ui + cls.nu] - torch.from_numpy(u_target).float().cuda()) ** 2).sum()
    loss.backward()
    gp, gl, gu = p.grad.cpu().numpy(), lo.grad.cpu().numpy(), hi.grad.cpu().numpy()
    cpu = CpuOSQP(plan, np.float64)
    f64 = lambda a: a.astype(np.float64)  # noqa: E731

    def loss_np(pv, lv, uv):
        xs = cpu.solve(pv, f64(b.a_values), f64(b.q), lv, uv, max_iter=6000)[0]
        return float(np.sum((xs[:, ui : ui + cls.nu] - u_target) ** 2))

    h = 1e-6
    P0, L0, U0 = f64(b.p_values), f64(b.l), f64(b.u)
    # x0 enters through l = u = -x0 on the first nx rows
    for r in range(cls.nx):
        Lp, Up, Lm, Um = L0.copy(), U0.copy(), L0.copy(), U0.copy()
        Lp[:, r] += h; Up[:, r] += h; Lm[:, r] -= h; Um[:, r] -= h
        fd = (loss_np(P0, Lp, Up) - loss_np(P0, Lm, Um)) / (2 * h)
        an = float(np.sum(gl[:, r] + gu[:, r]))
        assert abs(an - fd) <= 2e-3 * max(1.0, abs(fd)), (r, an, fd)
    # a diagonal entry of Q (first state weight, all stages share it per instance only through P entries)
    for k in (0, 5):
        Pp, Pm = P0.copy(), P0.copy()
        Pp[:, k] += h
        Pm[:, k] -= h
        fd = (loss_np(Pp, L0, U0) - loss_np(Pm, L0, U0)) / (2 * h)
        an = float(np.sum(gp[:, k]))
        assert abs(an - fd) <= 2e-3 * max(1.0, abs(fd)), (k, an, fd)


def test_adjoint_vs_reference_gradient_path(cuda_device):
    b, plan, comp = _setup(problems.SMALL, 6, seed=51)
    eng = comp.engine
    x, z, y, *_ = eng.solve(_t(b.p_values), _t(b.a_values), _t(b.q), _t(b.l), _t(b.u), keep_factor=True)
    rng = np.random.default_rng(9)
    dx = rng.standard_normal((6, plan.n)).astype(np.float32)
    got = eng.adjoint(eng.last_workspace, _t(b.p_values), _t(b.a_values), _t(b.l), _t(b.u), x, z, y, _t(dx), None)
    dq = got[0].cpu().numpy()
    X, Y = x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)
    errs = []
    for i in range(6):
        ref = adjoint_ref.adjoint(plan, b.p_values[i].astype(np.float64), b.a_values[i].astype(np.float64),
                                  b.l[i].astype(np.float64), b.u[i].astype(np.float64), X[i], Y[i],
                                  dx[i].astype(np.float64), np.zeros(plan.m))
        errs.append(_rel(dq[i], ref[0]))
    assert max(errs) < 5e-2, errs


def test_solve_with_objective_cotangent_and_shared_matrices(cuda_device):
    """Objective cotangent terms and broadcast (batch-1) P/A gradients sum over the batch."""
    import torch

    b, plan, comp = _setup(problems.SMALL, 8, seed=61)
    p = _t(b.p_values[:1]).requires_grad_(True)
    a = _t(b.a_values[:1]).requires_grad_(True)
    q = _t(b.q).requires_grad_(True)
    x, z, y, prim, dual, obj = comp.solve(p, a, q, _t(b.l), _t(b.u))
    obj.sum().backward()
    assert p.grad.shape == p.shape and a.grad.shape == a.shape
    # d obj / d q = x at the optimum (envelope theorem)
    np.testing.assert_allclose(q.grad.cpu().numpy(), x.detach().cpu().numpy(), rtol=2e-3, atol=2e-3)


def test_adjoint_residual_optional(cuda_device):
    """The differential QP's residual is formed only on request; the
    gradients are the same bits either way."""
    b, plan, comp = _setup(problems.SMALL, 12, seed=71, iters=40)
    eng = comp.engine
    args = [_t(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u)]
    x, z, y, *_ = eng.solve(*args, keep_factor=True)
    dx = _t(np.random.default_rng(3).standard_normal((12, plan.n)).astype(np.float32))
    plain = eng.adjoint(eng.last_workspace, args[0], args[1], args[3], args[4], x, z, y, dx, None)
    assert eng.last_adjoint_residual is None
    with_res = eng.adjoint(eng.last_workspace, args[0], args[1], args[3], args[4], x, z, y, dx, None, residual=True)
    for a, c in zip(plain, with_res):
        np.testing.assert_array_equal(a.cpu().numpy(), c.cpu().numpy())
    assert np.all(np.isfinite(eng.last_adjoint_residual.cpu().numpy()))
