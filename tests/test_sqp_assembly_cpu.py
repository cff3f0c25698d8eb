"""Sparse MPC QP assembly: the plan against the reference planner's fixtures,
and the assembly oracle against a dense reconstruction (no GPU needed).

Fixtures ``tests/golden/sqp_plan_*.npz`` come from the reference's own
``build_sparse_mpc_plan`` (``warpmpc/jax_sqp/sparse_mpc.py:532-691``) on the
synthetic stage descriptions of ``warpmpc_b200/sqp_problems.py``
(``tests/golden/make_golden.py``).
"""

import glob
import os

import numpy as np
import pytest

from oracle import assembly_ref
from warpmpc_b200 import problems, sqp_problems
from warpmpc_b200.jax_sqp import build_sparse_mpc_plan
from warpmpc_b200.jax_sqp.assembly import assembly_tables

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CLASSES = {"small": problems.SMALL,
           "quadrotor_n5": problems.MPCClass("quadrotor-n5", 12, 4, 5, 10.0, 2.0, 1.0, "quadrotor")}
FIX = sorted(glob.glob(os.path.join(GOLDEN, "sqp_plan_*.npz")))


def _eq(a, b, name):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and np.array_equal(a, b), name


@pytest.mark.parametrize("path", FIX, ids=[os.path.basename(p) for p in FIX])
def test_sparse_mpc_plan_matches_reference(path):
    g = np.load(path)
    name = os.path.basename(path)[len("sqp_plan_"):-4]
    prob = sqp_problems.make_problem(CLASSES[name])
    plan = build_sparse_mpc_plan(prob)
    for k in ("stage_var_dims", "param_dims", "constraint_dims"):
        _eq(np.asarray(getattr(plan, k)), g[k], k)
    for k in ("z_offsets", "param_offsets", "constraint_offsets", "representative_l", "representative_u"):
        _eq(getattr(plan, k), g[k], k)
    for k in ("p_pattern", "a_pattern"):
        _eq(getattr(plan, k).indices, g[k + "_indices"], k)
        _eq(getattr(plan, k).indptr, g[k + "_indptr"], k)
    for k in ("q_cols", "p_pos", "a_pos"):
        _eq(np.concatenate([getattr(a, k) for a in plan.assemblies]), g["asm_" + k], k)
        _eq([getattr(a, k).size for a in plan.assemblies], g["asm_" + k + "_counts"], k)
    for k in ("z_offset", "next_z_offset", "param_offset", "constraint_offset"):
        _eq([getattr(a, k) for a in plan.assemblies], g["asm_" + k], k)
    for k in g.files:
        if k.startswith("osqp_"):
            _eq(getattr(plan.osqp_plan, k[5:]), g[k], k)


def test_assembly_oracle_reconstructs_cost_and_constraints():
    import torch

    prob = sqp_problems.make_problem(problems.SMALL)
    plan = build_sparse_mpc_plan(prob)
    data = sqp_problems.make_data(problems.SMALL, 6, seed=2)
    gen = torch.Generator().manual_seed(0)
    z = torch.randn(6, int(plan.z_offsets[-1]), generator=gen)
    p = torch.randn(6, 4, generator=gen)
    vals = [[v.numpy() for v in s] for s in sqp_problems.evaluate_stages(prob, data, z, p)]
    pv, av, q, l, u, cost, g, lo, up = assembly_ref.assemble(plan, prob, vals)
    pr, pc = plan.p_pattern.indices, np.repeat(np.arange(plan.p_pattern.shape[1]), np.diff(plan.p_pattern.indptr))
    ar, ac = plan.a_pattern.indices, np.repeat(np.arange(plan.a_pattern.shape[1]), np.diff(plan.a_pattern.indptr))
    for i in range(6):
        P = np.zeros(plan.p_pattern.shape)
        P[pr, pc] = pv[i]
        P = P + np.triu(P, 1).T
        A = np.zeros(plan.a_pattern.shape)
        A[ar, ac] = av[i]
        zi = z[i].double().numpy()
        assert abs(0.5 * zi @ P @ zi - cost[i]) <= 1e-5 * (1 + abs(cost[i]))  # quadratic cost, zero constant
        np.testing.assert_allclose(P @ zi, q[i], rtol=1e-5, atol=1e-5)  # grad of a quadratic = P z
        np.testing.assert_allclose(A @ zi, g[i], rtol=1e-5, atol=1e-5)  # linear constraints: g = A z
    np.testing.assert_array_equal(l, lo - g)
    np.testing.assert_array_equal(u, up - g)


def test_assembly_tables_cover_every_stage_value_once():
    prob = sqp_problems.make_problem(problems.SMALL)
    plan = build_sparse_mpc_plan(prob)
    t = assembly_tables(plan, prob)
    offs = t["stage_offsets"]
    expect = sum(a.q_cols.size + a.p_pos.size + a.a_pos.size for a in plan.assemblies)
    assert t["add_src"].size == expect and t["add_ptr"][-1] == expect
    assert len(set(t["add_src"].tolist())) == expect  # no value added twice
    assert t["add_src"].max() < t["width"] and t["cost_src"].tolist() == offs[:, 0].tolist()
