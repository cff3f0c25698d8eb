"""Several problem classes in one persistent launch (wmpc_osqp_solve_persistent).

Each class keeps its own plan, factor and state; the launch walks every
class's instance tiles.  With a fixed iteration count every class's iterates
equal the float32 oracle bit for bit (the same arithmetic as a one-class
solve); with termination every instance stops on its own and the returned
iterate passes OSQP's residual test.
"""

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp, solve_classes

pytestmark = pytest.mark.gpu


def _problem(comp, b, warm=None):
    import torch

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return (comp.engine, t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u),
            None if warm is None else tuple(t(w) for w in warm))


def test_classes_one_launch_bitexact(cuda_device):
    specs = [(problems.QUADROTOR, 41), (problems.SMALL, 75), (problems.CARTPOLE, 33)]
    items, refs = [], []
    for k, (cls, batch) in enumerate(specs):
        b = problems.make_batch(cls, batch, seed=20 + k)
        plan = problems.make_plan(b)
        comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
        items.append(_problem(comp, b))
        refs.append(osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u))
    outs = solve_classes(items)
    for out, ref in zip(outs, refs):
        for name, g, r in zip(("x", "z", "y"), out[:3], ref[:3]):
            np.testing.assert_array_equal(g.cpu().numpy(), r, err_msg=name)


def test_classes_with_termination(cuda_device):
    specs = [(problems.SMALL, 64), (problems.QUADROTOR, 50)]
    items, plans, batches = [], [], []
    for k, (cls, batch) in enumerate(specs):
        b = problems.make_batch(cls, batch, seed=40 + k)
        settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 300})
        plan = problems.make_plan(b, settings)
        comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
        items.append(_problem(comp, b))
        plans.append(plan)
        batches.append(b)
    outs = solve_classes(items, check_termination=1)
    stopped_early = []
    for out, plan, b in zip(outs, plans, batches):
        x, z, y, prim, dual, obj, iters, status = (t.cpu().numpy() for t in out)
        p64, a64 = b.p_values.astype(np.float64), b.a_values.astype(np.float64)
        ax = osqp_ref.a_matvec(plan, a64, x.astype(np.float64))
        px = osqp_ref.p_matvec(plan, p64, x.astype(np.float64))
        aty = osqp_ref.at_matvec(plan, a64, y.astype(np.float64))
        eps_p = 1e-3 + 1e-3 * np.maximum(np.abs(ax).max(1), np.abs(z).max(1))
        eps_d = 1e-3 + 1e-3 * np.maximum(np.maximum(np.abs(px).max(1), np.abs(aty).max(1)), np.abs(b.q).max(1))
        passes = (prim <= eps_p * (1 + 1e-3)) & (dual <= eps_d * (1 + 1e-3))
        solved = (status & 1) != 0
        # SOLVED is the exact residual test of the returned iterate
        assert np.all(passes[solved])
        assert np.all((iters >= 1) & (iters <= 300))
        stopped_early.append(int(np.sum(iters < 300)))
        # stopping on the iterate-change test costs few instances their solution
        ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u)
        ref_ok = (ref[3] <= 1e-3) & (ref[4] <= 1e-3)
        assert solved.sum() >= 0.9 * ref_ok.sum(), (solved.sum(), ref_ok.sum())
    assert sum(stopped_early) > 0


def test_classes_warm_started_termination_is_sound(cuda_device):
    """Warm starts near a solution: an instance may stop at its first check,
    but only once its exact primal residual is within eps_abs (the kernel
    carries A x - z through the iterations), so the early stops keep their
    solutions -- in a closed loop the starting iterate is often already
    primal-infeasible by more than eps while barely moving."""
    specs = [(problems.SMALL, 64), (problems.QUADROTOR, 50)]
    items, plans, batches = [], [], []
    for k, (cls, batch) in enumerate(specs):
        b = problems.make_batch(cls, batch, seed=60 + k)
        settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 300})
        plan = problems.make_plan(b, settings)
        # start from the solution of a neighbouring problem (q and the bounds moved)
        rng = np.random.default_rng(70 + k)
        q0 = (b.q + 0.05 * rng.standard_normal(b.q.shape)).astype(np.float32)
        cold = osqp_ref.solve(plan, b.p_values, b.a_values, q0, b.l, b.u, max_iter=100)
        warm = tuple(np.asarray(w, dtype=np.float32) for w in cold[:3])
        comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
        items.append(_problem(comp, b, warm))
        plans.append(plan)
        batches.append((b, warm))
    outs = solve_classes(items, check_termination=1)
    for out, plan, (b, warm) in zip(outs, plans, batches):
        x, z, y, prim, dual, obj, iters, status = (t.cpu().numpy() for t in out)
        a64 = b.a_values.astype(np.float64)
        prim64 = np.abs(osqp_ref.a_matvec(plan, a64, x.astype(np.float64)) - z).max(1)
        early = iters < 300
        assert np.all(prim64[early] <= 1e-3 * 1.01), prim64[early].max()
        ref = osqp_ref.solve_warm_start(plan, b.p_values, b.a_values, b.q, b.l, b.u, *warm)
        ref_ok = (ref[3] <= 1e-3) & (ref[4] <= 1e-3)
        solved = (status & 1) != 0
        assert solved.sum() >= 0.9 * ref_ok.sum(), (solved.sum(), ref_ok.sum())
