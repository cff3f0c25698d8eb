"""Nonlinear SQP workload on the GPU: the rigid-body quadrotor RK4 model
kernel against the float64 oracle (values and finite-difference
Jacobians), one SQP step against the CPU pipeline of oracles fed the same
model values, SQP iterations that drive the dynamics residual down and replay
from a CUDA graph, and the gradient through the last QP against central
finite differences of converged float64 QP solves."""

import numpy as np
import pytest

from oracle import assembly_ref, line_search_ref, osqp_ref, quadrotor_ref
from warpmpc_b200 import quadrotor_sqp as qs

pytestmark = pytest.mark.gpu

LS = dict(g_max=1e-1, g_min=1e-3, gamma_c=1e-3, armijo_factor=1e-4, constraint_scale=0.1,
          cost_accept_uses_trial_cost=True)


def _random_z(batch, horizon, seed):
    rng = np.random.default_rng(seed)
    blocks = []
    for _ in range(horizon):
        x = np.concatenate([rng.uniform(-1, 1, (batch, 3)), rng.uniform(-0.4, 0.4, (batch, 3)),
                            rng.uniform(-1, 1, (batch, 3)), rng.uniform(-2, 2, (batch, 3))], 1)
        blocks += [x, rng.uniform(0.0, qs.U_MAX, (batch, qs.NU))]
    blocks.append(rng.uniform(-1, 1, (batch, qs.NX)))
    return np.concatenate(blocks, 1)


def test_model_kernel_matches_oracle(cuda_device):
    import torch

    batch, horizon = 64, 5
    z = _random_z(batch, horizon, 3)
    prob = qs.make_problem(horizon)
    ev = qs.Evaluator(prob, np.ones((batch, qs.NX)), np.ones((batch, qs.NU)), cuda_device)
    xn, jac = ev.dynamics(torch.from_numpy(z.astype(np.float32)).to(cuda_device), True)
    xn, jac = xn.cpu().numpy(), jac.cpu().numpy()
    cols, ptr = qs.jac_pattern()
    for k in range(horizon):
        x = z[:, 16 * k : 16 * k + 12].astype(np.float32).astype(np.float64)
        u = z[:, 16 * k + 12 : 16 * k + 16].astype(np.float32).astype(np.float64)
        want = quadrotor_ref.rk4(x, u)
        np.testing.assert_allclose(xn[k], want, rtol=0, atol=2e-6 * max(1.0, np.abs(want).max()))
        jfd = quadrotor_ref.rk4_jacobian_fd(x, u)
        for r in range(qs.NX):
            e = np.arange(ptr[r], ptr[r + 1] - 1)
            got = -jac[k][:, e]
            ref = jfd[:, r, cols[e]]
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5 * max(1.0, np.abs(ref).max()))
            np.testing.assert_array_equal(jac[k][:, ptr[r + 1] - 1], 1.0)
        # entries outside the pattern are zero in the oracle
        mask = np.zeros((qs.NX, 16), bool)
        for r in range(qs.NX):
            mask[r, cols[ptr[r] : ptr[r + 1] - 1]] = True
        assert np.abs(jfd[:, ~mask]).max() < 1e-9


def _setup(batch, horizon, seed, max_iter=25):
    data = qs.make_data(batch, seed)
    return qs.QuadrotorSQP(horizon, data, "cuda:0", iterations=5, max_iter=max_iter), data


def test_step_matches_oracle_pipeline(cuda_device):
    w, _ = _setup(32, 8, 1)
    z = qs.initial_guess(w.plan, w.x0)
    r = w.sqp.line_search_step(z, w.x0, None)
    host = lambda vals: [[v.cpu().numpy() for v in s] for s in vals]  # noqa: E731
    ev = w.evaluator
    lin = assembly_ref.assemble(w.plan, w.problem, host(ev(z, w.x0, False)))
    x, *_ = osqp_ref.solve(w.plan.osqp_plan, lin[0], lin[1], lin[2], lin[3], lin[4])
    np.testing.assert_array_equal(r.solve.direction.cpu().numpy(), x)
    d = r.solve.direction
    costs, viols = [], []
    steps = line_search_ref.make_step_lengths(0.5, 0.1).astype(np.float32)
    for step in steps:
        out = assembly_ref.assemble(w.plan, w.problem, host(ev(z + float(step) * d, w.x0, True)), values_only=True)
        costs.append(out[5])
        viols.append(line_search_ref.constraint_violation(out[7], out[6], out[8], 0.1))
    z_next, fin, bviol, armijo, res = line_search_ref.line_search_step(
        LS, steps, z.cpu().numpy(), x, lin[2], lin[7], lin[6], lin[8], lin[5], np.stack(costs),
        np.stack(viols).astype(np.float32))
    np.testing.assert_array_equal(r.line_search.step_length.cpu().numpy(), res[0])
    np.testing.assert_array_equal(r.z_next.cpu().numpy(), z_next)


def test_iterations_reduce_residual_and_graph_replays(cuda_device):
    import torch

    w, _ = _setup(64, 10, 2)

    def dyn_residual(zz):
        c, g, lo, up = w.sqp.evaluate_nlp(zz, w.x0)
        viol = torch.clamp(lo - g, min=0) + torch.clamp(g - up, min=0)
        return float(viol.abs().max())

    z0 = qs.initial_guess(w.plan, w.x0)
    v0 = dyn_residual(z0)
    z, _ = w.solve()
    assert dyn_residual(z) < 0.1 * v0
    eager = z.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        w.solve()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out, _ = w.solve()
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), eager.cpu().numpy())


def test_gradient_through_last_qp_matches_finite_differences(cuda_device):
    """Converged QP solves (forward and adjoint 2000 iterations) so that the
    adjoint's own convergence does not dominate; float64 oracle QPs for FD."""
    import torch

    from oracle.cpu_baseline import CpuOSQP

    batch, horizon = 8, 6
    w, data = _setup(batch, horizon, 5, max_iter=2000)
    w.sqp.qp.engine  # noqa: B018
    z, r = w.solve(keep_factor=True)
    ut = torch.full((batch, qs.NU), qs.U_HOVER * 1.1, device=cuda_device)
    gx0, gq, gr = (t.cpu().numpy().astype(np.float64) for t in w.gradient(z, r, ut))
    lin = [t.cpu().numpy().astype(np.float64) for t in r.solve.linearization[:5]]
    step = r.line_search.step_length.cpu().numpy().astype(np.float64)[:, None]
    z_lin = (z - r.line_search.step_length.reshape(-1, 1) * r.solve.direction).cpu().numpy().astype(np.float64)
    cpu = CpuOSQP(w.plan.osqp_plan, np.float64)
    ui = slice(qs.NX, qs.NX + qs.NU)
    utn = ut.cpu().numpy().astype(np.float64)

    def loss(p, q, l, u):
        d = cpu.solve(p, lin[1], q, l, u, max_iter=20000)[0]
        return np.sum((z_lin[:, ui] + step * d[:, ui] - utn) ** 2, axis=1)

    h = 1e-6
    p0, q0, l0, u0 = lin[0], lin[2], lin[3], lin[4]
    cols = [np.asarray(a.q_cols) for a in w.plan.assemblies]
    pos = [np.asarray(a.p_pos) for a in w.plan.assemblies]
    worst = 0.0
    for j in range(qs.NX):  # x0_j: l = u = x0 - x_lin0 on row j
        lp, up_, lm, um = l0.copy(), u0.copy(), l0.copy(), u0.copy()
        lp[:, j] += h; up_[:, j] += h; lm[:, j] -= h; um[:, j] -= h
        fd = (loss(p0, q0, lp, up_) - loss(p0, q0, lm, um)) / (2 * h)
        worst = max(worst, float(np.max(np.abs(gx0[:, j] - fd) / np.maximum(1e-3, np.abs(fd)))))
    for j in (0, 3, 9):  # Q_j: P diagonal entries and q = Q_j x_lin
        pp, pm, qp_, qm = p0.copy(), p0.copy(), q0.copy(), q0.copy()
        for k in range(horizon + 1):
            off = 16 * k
            pp[:, pos[k][j]] += h; pm[:, pos[k][j]] -= h
            qp_[:, cols[k][j]] += h * z_lin[:, off + j]; qm[:, cols[k][j]] -= h * z_lin[:, off + j]
        fd = (loss(pp, qp_, l0, u0) - loss(pm, qm, l0, u0)) / (2 * h)
        worst = max(worst, float(np.max(np.abs(gq[:, j] - fd) / np.maximum(1e-3, np.abs(fd)))))
    assert worst < 2e-2, worst


def test_solve_and_gradient_graph_replay(cuda_device):
    """The bench's nonlinear leg: the SQP iterations (last QP keeping its
    factorization) followed by the gradient, captured in one CUDA graph with
    the driver's one QP workspace, replay the eager results bit for bit."""
    import torch

    batch = 64
    w, _ = _setup(batch, 10, 3)
    ut = torch.full((batch, qs.NU), qs.U_HOVER * 1.1, device=cuda_device)
    z, r = w.solve(keep_factor=True)
    eager = [t.clone() for t in (z, *w.gradient(z, r, ut))]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        zz, rr = w.solve(keep_factor=True)
        w.gradient(zz, rr, ut)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        zg, rg = w.solve(keep_factor=True)
        grads = w.gradient(zg, rg, ut)
    g.replay()
    torch.cuda.synchronize()
    for got, want in zip((zg, *grads), eager):
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())
    del g
