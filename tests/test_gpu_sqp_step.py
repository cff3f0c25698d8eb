"""One SQP step with the filter line search on the GPU (SparseMPCSQP).

The step against a CPU pipeline of oracles on the same model values: the QP
direction equals the float32 OSQP oracle's bit for bit; the line search, fed
the same candidate evaluations, picks the same step and z_next = z + step d
matches.  Then: steps reduce the constraint violation, and a step captured in
a CUDA graph replays to the same bits as the eager step.
"""

import numpy as np
import pytest

from oracle import assembly_ref, line_search_ref, osqp_ref
from warpmpc_b200 import problems, sqp_problems
from warpmpc_b200.jax_sqp import SparseMPCSQP, build_sparse_mpc_plan

pytestmark = pytest.mark.gpu

LS = dict(g_max=1e-1, g_min=1e-3, gamma_c=1e-3, armijo_factor=1e-4, constraint_scale=0.1,
          cost_accept_uses_trial_cost=True)


def _setup(batch, seed):
    import torch

    cls = problems.SMALL
    prob = sqp_problems.make_problem(cls)
    plan = build_sparse_mpc_plan(prob)
    dev = torch.device("cuda", 0)
    ev = sqp_problems.make_evaluator(prob, sqp_problems.make_data(cls, batch, seed=seed), dev)
    sqp = SparseMPCSQP(prob, plan, ev, device=dev)
    gen = torch.Generator(device=dev).manual_seed(seed)
    params = torch.rand(batch, cls.nx, device=dev, generator=gen) * 2 - 1
    z = torch.zeros(batch, int(plan.z_offsets[-1]), device=dev)
    return prob, plan, ev, sqp, z, params


def test_step_matches_oracle_pipeline(cuda_device):
    import torch

    prob, plan, ev, sqp, z, params = _setup(48, 1)
    r = sqp.line_search_step(z, params, None)
    host = lambda vals: [[v.cpu().numpy() for v in s] for s in vals]  # noqa: E731
    lin = assembly_ref.assemble(plan, prob, host(ev(z, params, False)))
    x, *_ = osqp_ref.solve(plan.osqp_plan, lin[0], lin[1], lin[2], lin[3], lin[4])
    np.testing.assert_array_equal(r.solve.direction.cpu().numpy(), x)
    d = r.solve.direction
    costs, viols = [], []
    for step in line_search_ref.make_step_lengths(0.5, 0.1).astype(np.float32):
        out = assembly_ref.assemble(plan, prob, host(ev(z + float(step) * d, params, True)), values_only=True)
        costs.append(out[5])
        viols.append(line_search_ref.constraint_violation(out[7], out[6], out[8], 0.1))
    z_next, fin, bviol, armijo, res = line_search_ref.line_search_step(
        LS, line_search_ref.make_step_lengths(0.5, 0.1).astype(np.float32), z.cpu().numpy(), x, lin[2], lin[7],
        lin[6], lin[8], lin[5], np.stack(costs), np.stack(viols).astype(np.float32))
    np.testing.assert_array_equal(r.line_search.step_length.cpu().numpy(), res[0])
    np.testing.assert_array_equal(r.line_search.accepted.cpu().numpy(), res[4])
    np.testing.assert_array_equal(r.z_next.cpu().numpy(), z_next)
    assert bool(r.is_finite.all())


def test_steps_reduce_violation_and_graph_replays(cuda_device):
    import torch

    prob, plan, ev, sqp, z, params = _setup(64, 2)

    def violation(zz):
        c, g, lo, up = sqp.evaluate_nlp(zz, params)
        return float((torch.clamp(lo - g, min=0) ** 2 + torch.clamp(up - g, max=0) ** 2).sum(1).sqrt().max())

    v0 = violation(z)
    warm = None
    zz = z
    for _ in range(4):
        r = sqp.line_search_step(zz, params, warm)
        zz = r.z_next
        warm = (r.solve.direction, r.solve.z, r.solve.y)
    assert violation(zz) < 0.5 * v0
    # graph capture of one step from a fixed state; replay equals the eager step
    z_in = zz.clone()
    eager = sqp.line_search_step(z_in, params, None).z_next.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        sqp.line_search_step(z_in, params, None)  # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = sqp.line_search_step(z_in, params, None)
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.z_next.cpu().numpy(), eager.cpu().numpy())
