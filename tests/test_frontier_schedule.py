"""Frontier-slot schedules (host schedule of the next streaming-kernel form).

The schedule renames the work-vector rows to slots that hold only what a
sweep still reads; right-hand sides and forward results travel through the
stages instead.  The CPU replay runs that form with every index bounds-checked
and the releases of each backward chunk deferred by the schedule's lag (the
most a release may trail the sweep): its iterates equal the oracle's bit for
bit, cold and warm started, so no slot is reused while something still reads
it.  The streaming kernel runs this form when a problem is created with
WMPC_STREAM_FRONTIER=1 (GPU parity in test_gpu_frontier.py).
"""

import os
import sys

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import problems
from warpmpc_b200.schedule import stream_schedule

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import stream_sim  # noqa: E402

FRONTIER = (16, 16, 12, 16, 4)
FRONTIER_24 = (24, 24, 16, 24, 4)  # the library's default chunk targets


@pytest.mark.parametrize("cls,iters", [(problems.SMALL, 4), (problems.CARTPOLE, 3),
                                       (problems.MPCClass("q5", 12, 4, 5, 10.0, 2.0, 1.0, "quadrotor"), 3)],
                         ids=["small", "cartpole", "quadrotor_n5"])
@pytest.mark.parametrize("lag", [None, 1])
@pytest.mark.parametrize("targets", [FRONTIER, FRONTIER_24], ids=["chunks16", "chunks24"])
def test_frontier_replay_bitexact(cls, iters, lag, targets):
    b = problems.make_batch(cls, 6, seed=31)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan, targets=targets)
    assert 0 < sched["frontier_slots"] < plan.qdldl_plan.n and sched["frontier_lag"] == 4
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=iters, lag=lag)
    ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=iters)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)


def test_frontier_replay_warm_start():
    b = problems.make_batch(problems.SMALL, 8, seed=7)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan, targets=FRONTIER)
    x, z, y = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=3)[:3]
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, x0=x, z0=z, y0=y, max_iter=3)
    ref = osqp_ref.solve_warm_start(plan, b.p_values, b.a_values, b.q, b.l, b.u, x, z, y, max_iter=3)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)


def test_frontier_slots_shrink_the_work_vector():
    """Slots needed against rows for the benchmark patterns: the quadrotor's
    work vector drops from 1358 rows to about 500."""
    for cls, most in ((problems.SMALL, 0.6), (problems.CARTPOLE, 0.5), (problems.QUADROTOR, 0.45)):
        plan = problems.make_plan(problems.make_batch(cls, 2, seed=0))
        sched = stream_schedule(plan, targets=FRONTIER)
        assert sched["frontier_slots"] <= most * plan.qdldl_plan.n, (cls.name, sched["frontier_slots"])


def test_frontier_needs_no_offload():
    plan = problems.make_plan(problems.make_batch(problems.SMALL, 2, seed=0))
    with pytest.raises(NotImplementedError):
        stream_schedule(plan, targets=(16, 16, 12, 16, 4 | 1))


def test_frontier_replay_detects_releases_later_than_the_schedule_allows():
    """Control: releases trailing the sweep by more chunks than the schedule
    reserved slots for read reused slots, and the iterates change."""
    b = problems.make_batch(problems.SMALL, 6, seed=31)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan, targets=FRONTIER)
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=3, lag=8)
    ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=3)
    assert not all(np.array_equal(g, r) for g, r in zip(got, ref[:3]))


FRONTIER_COPIES = (16, 16, 12, 16, 4 | 8)


@pytest.mark.parametrize("cls,iters", [(problems.SMALL, 4), (problems.CARTPOLE, 3),
                                       (problems.MPCClass("q5", 12, 4, 5, 10.0, 2.0, 1.0, "quadrotor"), 3)],
                         ids=["small", "cartpole", "quadrotor_n5"])
def test_frontier_copies_replay_bitexact(cls, iters):
    """Rows without entries copied from the stage into their slots at their
    chunk's start (no unit swept for them): same bits as the oracle, cold and
    warm, with the releases deferred by the schedule's lag; the forward
    sweep has fewer units and no more slots than with copy units."""
    b = problems.make_batch(cls, 6, seed=37)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan, targets=FRONTIER_COPIES)
    base = stream_schedule(plan, targets=FRONTIER)
    assert int(np.sum(sched["fchunk_units"])) < int(np.sum(base["fchunk_units"]))
    assert sched["frontier_slots"] <= base["frontier_slots"] + 2
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=iters)
    ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=iters)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)
    x, z, y = ref[:3]
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, x0=x, z0=z, y0=y, max_iter=iters)
    ref = osqp_ref.solve_warm_start(plan, b.p_values, b.a_values, b.q, b.l, b.u, x, z, y, max_iter=iters)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)


@pytest.mark.parametrize("bits", [0, 3, 4, 4 | 8], ids=["plain", "plain_offload", "frontier", "frontier_copies"])
def test_schedule_replay_random_patterns(bits):
    """Random sparse QPs (box, equality, one-sided and free rows) under small
    chunk targets, so that most rows sit near a chunk edge: the replay of the
    plain form (with and without releaser offload) and of the frontier form
    (copy units or copy lists) equals the oracle bit for bit on every
    pattern."""
    import scipy.sparse as sps

    from warpmpc_b200.jax_osqp import OSQPSettings
    from warpmpc_b200.jax_osqp.planning import build_osqp_plan

    rng = np.random.default_rng(71)
    for trial in range(6):
        n, m = int(rng.integers(4, 30)), int(rng.integers(3, 40))
        p = sps.random(n, n, density=float(rng.uniform(0.05, 0.3)), random_state=int(rng.integers(1 << 30)))
        p = sps.triu(sps.csc_matrix(p @ p.T + sps.eye(n)), format="csc")
        a = sps.csc_matrix(sps.random(m, n, density=float(rng.uniform(0.1, 0.4)),
                                      random_state=int(rng.integers(1 << 30))) + sps.eye(m, n))
        a.sum_duplicates()
        a.sort_indices()
        kind = rng.integers(0, 4, m)  # 0 box, 1 equality, 2 lower only, 3 free
        l = np.where(kind == 3, -1e30, rng.standard_normal(m) - 1.0)
        u = np.where(kind == 2, 1e30, np.where(kind == 1, l, l + rng.uniform(0.1, 2.0, m)))
        u = np.where(kind == 3, 1e30, u)
        plan = build_osqp_plan(p, a, l, u, OSQPSettings(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=4, rho_is_vec=True))
        targets = (4, 4, 3, 4, bits)
        sched = stream_schedule(plan, targets=targets)
        B = 5
        f32 = np.float32
        pv = (p.data[None, :] * rng.uniform(0.5, 1.5, (B, p.nnz))).astype(f32)
        av = (a.data[None, :] * rng.uniform(0.5, 1.5, (B, a.nnz))).astype(f32)
        q = rng.standard_normal((B, n)).astype(f32)
        lb = np.broadcast_to(l, (B, m)).astype(f32)
        ub = np.broadcast_to(u, (B, m)).astype(f32)
        got = stream_sim.replay(plan, sched, pv, av, q, lb, ub, max_iter=4)
        ref = osqp_ref.solve(plan, pv, av, q, lb, ub, max_iter=4)
        for name, g, r in zip("xzy", got, ref[:3]):
            np.testing.assert_array_equal(g, r, err_msg=f"trial {trial} ({n}x{m}): {name}")


@pytest.mark.parametrize("cls", [problems.SMALL, problems.CARTPOLE, problems.QUADROTOR],
                         ids=["small", "cartpole", "quadrotor"])
@pytest.mark.parametrize("targets", [FRONTIER, FRONTIER_24, FRONTIER_COPIES], ids=["chunks16", "chunks24", "copies"])
def test_frontier_release_records_close_each_backward_block(cls, targets):
    """The frontier-form producer copies a backward chunk's release records
    into its S stage as the last 4 nrel words of the chunk's meta block (one
    16-byte-aligned bulk copy) and the rest of the block into the L stage:
    the records must be exactly those words, in release order, each naming
    its slot and its permuted KKT index, and the rest must stay 16-byte
    aligned."""
    plan = problems.make_plan(problems.make_batch(cls, 2, seed=0))
    sched = stream_schedule(plan, targets=targets)
    slots = int(sched["frontier_slots"])
    assert slots > 0
    meta, u_perm = np.asarray(sched["meta"]), np.asarray(sched["u_perm"])
    for ch in range(int(sched["n_chunks"])):
        off, words = int(sched["meta_off"][ch]), int(sched["meta_words"][ch])
        m = meta[off : off + words]
        nrel, u0 = int(sched["chunk_nrel"][ch]), int(sched["chunk_u0"][ch])
        assert m[2] == nrel and m[4] == u0 and off % 4 == 0
        lead = words - 4 * nrel
        assert lead % 4 == 0 and lead >= 8
        rec = m[lead:].reshape(nrel, 4)
        np.testing.assert_array_equal(rec[:, 3], u_perm[u0 : u0 + nrel])
        assert np.all(rec[:, 0] % 128 == 0) and np.all((rec[:, 0] >= 0) & (rec[:, 0] < slots * 128))
