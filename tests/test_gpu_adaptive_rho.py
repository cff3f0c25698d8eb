"""rho adaptation on the GPU (per instance; the per-call kernels and the
streaming persistent path) against the oracle's restatement of the same
rule: iterates bit for bit, the same final rho and the same number of rho
changes (refactorizations) per instance.  The
reference has no rho adaptation (solver.py:587-588 rejects adaptive_rho);
the rule is OSQP's residual balancing (Stellato et al. 2020, sec. 5.2)."""

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["plain", "persistent"])
@pytest.mark.parametrize("cls", [problems.SMALL, problems.QUADROTOR], ids=lambda c: c.name)
def test_adaptive_rho_matches_oracle(cuda_device, cls, mode):
    import torch

    b = problems.make_batch(cls, 48, seed=17)
    settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 60, "adaptive_rho": True,
                               "adaptive_rho_interval": 10})
    plan = problems.make_plan(b, settings)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode=mode)
    assert comp.engine.mode == mode
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


@pytest.mark.parametrize("frontier", ["0", "1"])
def test_adaptive_rho_persistent_many_tiles(cuda_device, monkeypatch, frontier):
    """The streaming path over more tiles than SMs (several tiles per CTA, the
    tiles whose instances keep their rho skip the refactorization), both
    schedule forms, warm-started, against the per-call kernels: the same
    bits, rho and refactor counts."""
    import torch

    from warpmpc_b200 import native

    monkeypatch.setenv("WMPC_STREAM_FRONTIER", frontier)
    cls = problems.CARTPOLE
    n = 400 * 32 + 7
    b = problems.make_batch(cls, n, seed=37)
    settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 30, "adaptive_rho": True,
                               "adaptive_rho_interval": 8, "adaptive_rho_tolerance": 3.0})
    plan = problems.make_plan(b, settings)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    rng = np.random.default_rng(5)
    warm = [t(rng.standard_normal((n, k)).astype(np.float32) * 0.05) for k in (plan.n, plan.m, plan.m)]
    out = {}
    for mode in ("plain", "persistent"):
        comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode=mode)
        assert comp.engine.mode == mode
        got = comp.solve_warm_start(t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u), *warm)
        torch.cuda.synchronize()
        if mode == "persistent":
            assert native.stream_last_launch()["form"] == ("frontier" if frontier == "1" else "plain")
        out[mode] = ([o.cpu().numpy() for o in got[:3]], comp.engine.last_rho.cpu().numpy(),
                     comp.engine.last_rho_updates.cpu().numpy())
    (xp, rp, up), (xs, rs, us) = out["plain"], out["persistent"]
    for name, g, r in zip(("x", "z", "y"), xs, xp):
        np.testing.assert_array_equal(g, r, err_msg=name)
    np.testing.assert_array_equal(rs, rp)
    np.testing.assert_array_equal(us, up)
    assert 0 < (up > 0).sum() < n  # some instances changed rho, some kept it
