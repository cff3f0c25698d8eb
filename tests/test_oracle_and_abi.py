"""CPU checks of the oracle restatements and of the C ABI library.

* the C restatement (oracle/c/osqp_cpu.c) equals the NumPy restatement bit
  for bit (float32), and the float64 factor/solve solves the dense system;
* the library loads and exports every entry point declared in
  include/warpmpc_b200.h (no compute calls: this host has no GPU);
* the host-built streaming schedule, replayed on the CPU with the kernel's
  exact addressing (tests/stream_sim.py), is bit-exact with the oracle.
"""

import os
import re

import numpy as np
import pytest

from oracle import osqp_ref, qdldl_ref
from warpmpc_b200 import native, problems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _built():
    from warpmpc_b200 import build

    build.build()


def test_c_oracle_matches_numpy_oracle():
    from oracle.cpu_baseline import CpuOSQP

    for cls in (problems.SMALL, problems.CARTPOLE):
        b = problems.make_batch(cls, 12, seed=2)
        plan = problems.make_plan(b)
        got = CpuOSQP(plan).solve(b.p_values, b.a_values, b.q, b.l, b.u, threads=3)
        ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u)
        for g, r in zip(got[:5], ref[:5]):
            np.testing.assert_array_equal(g, r)
        np.testing.assert_allclose(got[5], ref[5], rtol=1e-5)


def test_oracle_float64_solves_kkt():
    b = problems.make_batch(problems.SMALL, 3, seed=4)
    plan = problems.make_plan(b)
    kkt = osqp_ref.assemble_kkt_values(plan, b.p_values.astype(np.float64), b.a_values.astype(np.float64))
    qp = plan.qdldl_plan
    rhs = np.random.default_rng(0).standard_normal((qp.n, 1))
    for i in range(3):
        lx, d, dinv = qdldl_ref.factor(qp, kkt[i][:, None])
        x = qdldl_ref.solve(qp, lx, dinv, rhs)
        assert np.max(np.abs(qdldl_ref.dense_kkt(qp, kkt[i]) @ x - rhs)) < 1e-9


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "warpmpc_b200.h")).read()
    declared = set(re.findall(r"\b(wmpc_[a-z0-9_]+)\s*\(", header))
    lib = native.lib()
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert declared >= set(native.SIGNATURES), set(native.SIGNATURES) - declared
    assert "sm_100a" in native.version()


def test_invalid_arguments_fail_cleanly():
    import ctypes

    lib = native.lib()
    assert lib.wmpc_plan_create(None, 0, None) == native.WMPC_ERR_INVALID_ARGUMENT
    assert b"null" in lib.wmpc_last_error_string()
    assert lib.wmpc_osqp_solve(None, None, None, None, None, 0, 0, None, 0, None) == native.WMPC_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("offload", [0, 1, 2, 3])
@pytest.mark.parametrize("cls", [problems.SMALL, problems.CARTPOLE], ids=lambda c: c.name)
def test_stream_schedule_replay_warm_start(cls, offload):
    """Warm start: the first right-hand side is non-zero everywhere, so every
    coefficient the first pass reads must have been copied into its stage."""
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    import stream_sim
    from oracle import osqp_ref
    from warpmpc_b200.schedule import stream_schedule

    b = problems.make_batch(cls, 8, seed=7)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan, targets=(16, 16, 12, 16, offload))
    x, z, y = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=3)[:3]
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, x0=x, z0=z, y0=y, max_iter=3)
    ref = osqp_ref.solve_warm_start(plan, b.p_values, b.a_values, b.q, b.l, b.u, x, z, y, max_iter=3)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)


@pytest.mark.parametrize("cls", [problems.SMALL, problems.CARTPOLE], ids=lambda c: c.name)
def test_stream_schedule_replay_bitexact(cls):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import stream_sim

    from warpmpc_b200.schedule import stream_schedule

    b = problems.make_batch(cls, 6, seed=13)
    plan = problems.make_plan(b)
    sched = stream_schedule(plan)
    got = stream_sim.replay(plan, sched, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=4)
    ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u, max_iter=4)
    for g, r in zip(got, ref[:3]):
        np.testing.assert_array_equal(g, r)
    # chunk invariants the kernel relies on
    q = plan.qdldl_plan
    assert sched["chunk_off"][-1] == sched["blen"] == 128 * sched["chunk_units"].sum() + 32 * q.n
    assert sched["fchunk_off"][-1] == sched["flen"] == 128 * sched["fchunk_units"].sum()
    # every L entry once in each stream (entries of rows the releaser solves forward sit in the
    # backward stream a second time), every other slot padding
    n_pre = int((sched["proc_foff"] < 0).sum())
    assert 4 * sched["chunk_units"].sum() == q.nnz_l + n_pre + sched["pad_boff"].size
    assert 4 * sched["fchunk_units"].sum() == q.nnz_l - n_pre + sched["pad_foff"].size
    assert np.unique(sched["proc_boff"]).size == q.nnz_l and np.unique(sched["proc_foff"]).size == q.nnz_l
    assert sorted(sched["u_perm"].tolist()) == list(range(plan.qdldl_plan.n))


def test_multiclass_entry_rejects_bad_arguments():
    """wmpc_osqp_solve_persistent validates before touching a device."""
    import ctypes

    lib = native.lib()
    null = ctypes.POINTER(ctypes.c_void_p)()
    rc = lib.wmpc_osqp_solve_persistent(null, None, None, 1, null, None, None)
    assert rc != 0 and b"null" in lib.wmpc_last_error_string()
    handles = (ctypes.c_void_p * 1)(None)
    opts = (native.OsqpOptions * 1)()
    data = (native.OsqpBatch * 1)()
    ws = (ctypes.c_void_p * 1)(None)
    wsb = (ctypes.c_size_t * 1)(0)
    rc = lib.wmpc_osqp_solve_persistent(handles, opts, data, 7, ws, wsb, None)
    assert rc != 0 and b"n_classes" in lib.wmpc_last_error_string()
