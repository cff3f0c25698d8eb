"""rho adaptation on the GPU (per instance, plain mode) against the oracle's
restatement of the same rule: iterates bit for bit, the same final rho and
the same number of rho changes (refactorizations) per instance.  The
reference has no rho adaptation (solver.py:587-588 rejects adaptive_rho);
the rule is OSQP's residual balancing (Stellato et al. 2020, sec. 5.2)."""

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cls", [problems.SMALL, problems.QUADROTOR], ids=lambda c: c.name)
def test_adaptive_rho_matches_oracle(cuda_device, cls):
    import torch

    b = problems.make_batch(cls, 48, seed=17)
    settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 60, "adaptive_rho": True,
                               "adaptive_rho_interval": 10})
    plan = problems.make_plan(b, settings)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    assert comp.engine.mode == "plain"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got = [o.cpu().numpy() for o in comp.solve(t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u))]
    rho = comp.engine.last_rho.cpu().numpy()
    upd = comp.engine.last_rho_updates.cpu().numpy()
    ref = osqp_ref.solve_adaptive(plan, b.p_values, b.a_values, b.q, b.l, b.u)
    for name, g, r in zip(("x", "z", "y"), got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r, err_msg=name)
    np.testing.assert_array_equal(rho, ref[6])
    np.testing.assert_array_equal(upd, ref[7])
    assert upd.sum() > 0  # the rule did change rho somewhere
    for g, r in zip(got[3:], ref[3:6]):
        assert np.max(np.abs(g - r)) <= 1e-4 * max(1.0, float(np.max(np.abs(r))))


def test_adaptive_rho_shared_matrices_and_warm_start(cuda_device):
    """P and A shared by the batch (batch 1) still factor per instance once rho differs."""
    import torch

    b = problems.make_batch(problems.SMALL, 24, seed=29)
    settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 40, "adaptive_rho": True,
                               "adaptive_rho_interval": 7, "adaptive_rho_tolerance": 2.0})
    plan = problems.make_plan(b, settings)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    rng = np.random.default_rng(3)
    warm = [rng.standard_normal((24, k)).astype(np.float32) * 0.1 for k in (plan.n, plan.m, plan.m)]
    got = comp.solve_warm_start(t(b.p_values[:1]), t(b.a_values[:1]), t(b.q), t(b.l), t(b.u), *[t(w) for w in warm])
    got = [o.cpu().numpy() for o in got]
    ref = osqp_ref.solve_adaptive(plan, b.p_values[:1], b.a_values[:1], b.q, b.l, b.u, warm=warm)
    for name, g, r in zip(("x", "z", "y"), got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r, err_msg=name)
    np.testing.assert_array_equal(comp.engine.last_rho_updates.cpu().numpy(), ref[7])
