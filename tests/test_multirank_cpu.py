"""Multi-rank host logic on CPU: two gloo ranks, each solving its own instances.

Covers what ``bench.py --gpus N`` does besides the kernels: every rank builds
the same plan from the shared representative instance (checked by digest),
solves its own seeded instances, and the job reports the max step time and
the summed converged count.  Solves here go through the oracle (CPU only).
"""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from warpmpc_b200 import multirank, problems  # noqa: E402

BATCH = 6
RES_TOL = 1e-3


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _converged(plan, b) -> int:
    from oracle import osqp_ref

    x, z, y, prim, dual, obj = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u)
    return int(np.sum((prim <= RES_TOL) & (dual <= RES_TOL)))


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    env = multirank.rank_env()
    dev = multirank.init(env, "gloo", timeout_s=60.0)
    try:
        if mode == "solve":
            b0 = problems.make_batch(problems.SMALL, 1, seed=1000)
            plan = problems.make_plan(b0)
            multirank.check_plans_agree(plan, env, dev)
            b = problems.make_batch(problems.SMALL, BATCH, seed=multirank.instance_seed(1000, env.rank))
            ok = _converged(plan, b)
            total = multirank.sum_over_ranks(ok, env, dev)
            slowest = multirank.max_over_ranks(10.0 + env.rank, env, dev)
            multirank.barrier(env)
            q.put((rank, "ok", ok, total, slowest))
        elif mode == "mismatch":
            b0 = problems.make_batch(problems.SMALL, 1, seed=1000 + env.rank)  # rank 1 builds another plan
            plan = problems.make_plan(b0)
            try:
                multirank.check_plans_agree(plan, env, dev)
                q.put((rank, "agreed", 0, 0, 0))
            except RuntimeError as exc:
                q.put((rank, "raised", str(exc), 0, 0))
    finally:
        multirank.finalize(env)


def _spawn(world, mode):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(world):
            item = q.get(timeout=240)
            results[item[0]] = item[1:]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return results


def test_shard_bounds_cover_exactly():
    for total in (0, 1, 7, 65536, 131071):
        for world in (1, 2, 3, 8):
            spans = [multirank.shard_bounds(total, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        multirank.shard_bounds(10, 2, 2)


def test_plan_digest_is_deterministic_and_sensitive():
    b0 = problems.make_batch(problems.SMALL, 1, seed=1000)
    d1 = multirank.plan_digest(problems.make_plan(b0))
    d2 = multirank.plan_digest(problems.make_plan(b0))
    d3 = multirank.plan_digest(problems.make_plan(problems.make_batch(problems.SMALL, 1, seed=1001)))
    assert d1 == d2 and d1 != d3


def test_two_ranks_weak_scaling_totals():
    res = _spawn(2, "solve")
    b0 = problems.make_batch(problems.SMALL, 1, seed=1000)
    plan = problems.make_plan(b0)
    expect = [_converged(plan, problems.make_batch(problems.SMALL, BATCH, seed=multirank.instance_seed(1000, r)))
              for r in range(2)]
    for r in range(2):
        status, ok, total, slowest = res[r]
        assert status == "ok"
        assert ok == expect[r]
        assert total == sum(expect)
        assert slowest == 11.0


def test_two_ranks_detect_plan_mismatch():
    res = _spawn(2, "mismatch")
    assert {v[0] for v in res.values()} == {"raised"}
