"""The streaming kernel's frontier form on the GPU vs the oracle.

With ``WMPC_STREAM_FRONTIER=1`` a compiled problem carries the frontier-slot
schedule: the work vector holds only what a sweep still reads, the
right-hand sides and forward results travel through per-tile vectors and the
stages.  Fixed-iteration solves then run that form; their iterates must equal
the oracle's bit for bit (the arithmetic and its order are unchanged).  The
quadrotor pattern uses 12-unit chunks so that two CTAs fit an SM.
"""

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp

pytestmark = pytest.mark.gpu

QUAD_KNOBS = {"WMPC_STREAM_UNITS": "12", "WMPC_STREAM_COLS": "12", "WMPC_STREAM_REL": "8",
              "WMPC_STREAM_FUNITS": "12"}


def _compile(monkeypatch, plan, knobs):
    monkeypatch.setenv("WMPC_STREAM_FRONTIER", "1")
    for k, v in knobs.items():
        monkeypatch.setenv(k, v)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    info = comp.engine.stream_info()
    assert info["streaming"] and 0 < info["frontier_slots"] < info["n"], info
    return comp


def _run(comp, b, warm=None):
    import torch

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    if warm is None:
        out = comp.solve(t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u))
    else:
        out = comp.solve_warm_start(t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u), *[t(w) for w in warm])
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("cls,batch,knobs", [(problems.SMALL, 9500, {}), (problems.CARTPOLE, 700, {}),
                                             (problems.QUADROTOR, 4801, QUAD_KNOBS)],
                         ids=["small", "cartpole", "quadrotor"])
def test_frontier_form_bitexact(cuda_device, monkeypatch, cls, batch, knobs):
    """Many tiles (two CTAs per SM where they fit), a partial last tile."""
    from oracle.cpu_baseline import CpuOSQP

    b = problems.make_batch(cls, batch, seed=23)
    plan = problems.make_plan(b)
    comp = _compile(monkeypatch, plan, knobs)
    got = _run(comp, b)
    ref = CpuOSQP(plan).solve(b.p_values, b.a_values, b.q, b.l, b.u)
    for name, g, r in zip(("x", "z", "y"), got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r, err_msg=name)
    assert not np.any(comp.engine.last_status.cpu().numpy() & 8)


def test_frontier_form_warm_start(cuda_device, monkeypatch):
    b = problems.make_batch(problems.CARTPOLE, 70, seed=4)
    plan = problems.make_plan(b)
    comp = _compile(monkeypatch, plan, {})
    rng = np.random.default_rng(2)
    warm = tuple((rng.standard_normal((70, k)) * 0.1).astype(np.float32) for k in (plan.n, plan.m, plan.m))
    got = _run(comp, b, warm=warm)
    ref = osqp_ref.solve_warm_start(plan, b.p_values, b.a_values, b.q, b.l, b.u, *warm)
    for g, r in zip(got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r)


@pytest.mark.parametrize("cls,batch", [(problems.SMALL, 40), (problems.CARTPOLE, 300)], ids=["small", "cartpole"])
def test_frontier_form_termination_checks(cuda_device, monkeypatch, cls, batch):
    """Checked solves in the frontier form (unscale factors from the index
    table, the second releaser following the stop decisions): the same
    iterates, iteration counts and status as the plain form's checked solve,
    cold and warm."""
    import torch

    from warpmpc_b200 import native

    b = problems.make_batch(cls, batch, seed=3)
    plan = problems.make_plan(b, OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 60}))
    comp = _compile(monkeypatch, plan, {})
    monkeypatch.setenv("WMPC_STREAM_FRONTIER", "0")
    plain = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    args = [t(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u)]
    rng = np.random.default_rng(8)
    for warm in (None, tuple(t(rng.standard_normal((batch, k)).astype(np.float32) * 0.1)
                             for k in (plan.n, plan.m, plan.m))):
        got = comp.engine.solve(*args, warm=warm, check_termination=5)
        assert native.stream_last_launch()["form"] == "frontier"
        iters = comp.engine.last_iters.cpu().numpy()
        status = comp.engine.last_status.cpu().numpy()
        want = plain.engine.solve(*args, warm=warm, check_termination=5)
        assert native.stream_last_launch()["form"] == "plain"
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g.cpu().numpy(), w.cpu().numpy())
        np.testing.assert_array_equal(iters, plain.engine.last_iters.cpu().numpy())
        np.testing.assert_array_equal(status, plain.engine.last_status.cpu().numpy())
        assert iters.min() < 60  # some instances stopped early


def test_frontier_beside_plain_schedule(cuda_device, monkeypatch):
    """WMPC_STREAM_FRONTIER=2 (the default) builds both schedules.  Solves of
    more tiles than SMs run the frontier form where it fits two CTAs per SM and
    the plain form does not (the quadrotor pattern), checked solves included.
    Iterates bit-exact against the oracle, and the checked solve equal to a
    plain-only problem's, iteration counts included."""
    import torch
    from oracle.cpu_baseline import CpuOSQP

    b = problems.make_batch(problems.QUADROTOR, 4801, seed=29)
    plan = problems.make_plan(b)
    monkeypatch.setenv("WMPC_STREAM_FRONTIER", "2")
    both = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    assert both.engine.stream_info()["frontier_slots"] > 0
    monkeypatch.setenv("WMPC_STREAM_FRONTIER", "0")
    plain = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    assert plain.engine.stream_info()["frontier_slots"] == 0
    got = _run(both, b)
    ref = CpuOSQP(plan).solve(b.p_values, b.a_values, b.q, b.l, b.u)
    for name, g, r in zip(("x", "z", "y"), got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r, err_msg=name)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    args = [t(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u)]
    checked = both.engine.solve(*args, check_termination=5)
    iters_both = both.engine.last_iters.cpu().numpy()
    want = plain.engine.solve(*args, check_termination=5)
    for g, w in zip(checked, want):
        np.testing.assert_array_equal(g.cpu().numpy(), w.cpu().numpy())
    np.testing.assert_array_equal(iters_both, plain.engine.last_iters.cpu().numpy())
