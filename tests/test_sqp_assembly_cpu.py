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


class _RandomStage:
    """A stage description with random local sparsity and bound types."""

    def __init__(self, rng, z_dim, next_z_dim, param_dim, constraint_dim):
        self.has_next = next_z_dim > 0
        self.z_dim, self.next_z_dim, self.param_dim, self.constraint_dim = z_dim, next_z_dim, param_dim, constraint_dim
        w = z_dim + next_z_dim
        self.grad_cols = np.sort(rng.choice(w, size=int(rng.integers(1, w + 1)), replace=False)).astype(np.int32)
        k = int(rng.integers(1, 2 * w))
        self.hess_rows = rng.integers(0, w, k).astype(np.int32)  # either triangle, repeats allowed
        self.hess_cols = rng.integers(0, w, k).astype(np.int32)
        kj = int(rng.integers(0, 3 * max(constraint_dim, 1))) if constraint_dim else 0
        self.jac_rows = rng.integers(0, max(constraint_dim, 1), kj).astype(np.int32)
        self.jac_cols = rng.integers(0, w, kj).astype(np.int32)
        self._kind = rng.integers(0, 4, constraint_dim)  # box, equality, lower only, free

    def value_function(self, z, *rest):
        fill = float(z[0]) if len(z) else 0.0
        lo = np.where(self._kind == 3, -1e30, fill - 1.0)
        up = np.where(self._kind == 2, 1e30, np.where(self._kind == 1, lo, fill + 1.0))
        up = np.where(self._kind == 3, 1e30, up)
        return 0.0, np.zeros(self.constraint_dim), lo, up


def test_live_reference_sparse_mpc_plans_random():
    """build_sparse_mpc_plan against the reference's on random stage patterns
    (where the reference tree exists)."""
    from oracle import ref_import

    if not ref_import.available():
        pytest.skip("reference checkout not present (fixtures cover this case)")
    from warpmpc_b200.jax_qdldl.amd import amd_order
    from warpmpc_b200.jax_sqp import SparseMPCProblem

    ref_import.PERMUTATION_PROVIDER = amd_order
    sm = ref_import.load_sqp()
    rng = np.random.default_rng(12)
    for trial in range(6):
        n_st = int(rng.integers(2, 6))
        dims = [int(rng.integers(1, 5)) for _ in range(n_st)]
        stages = [_RandomStage(rng, dims[i], dims[i + 1] if i + 1 < n_st else 0, int(rng.integers(0, 3)),
                               int(rng.integers(0, 4))) for i in range(n_st)]
        ref = sm.build_sparse_mpc_plan(sm.SparseMPCProblem(stages=tuple(stages)))
        mine = build_sparse_mpc_plan(SparseMPCProblem(tuple(stages)))
        for k in ("z_offsets", "param_offsets", "constraint_offsets", "representative_l", "representative_u"):
            _eq(getattr(mine, k), getattr(ref, k), f"{trial} {k}")
        for k in ("p_pattern", "a_pattern"):
            _eq(getattr(mine, k).indices, getattr(ref, k).indices, f"{trial} {k}")
            _eq(getattr(mine, k).indptr, getattr(ref, k).indptr, f"{trial} {k}")
        for a, b in zip(mine.assemblies, ref.assemblies):
            for k in ("q_cols", "p_pos", "a_pos"):
                _eq(getattr(a, k), getattr(b, k), f"{trial} {k}")
            for k in ("z_offset", "next_z_offset", "param_offset", "constraint_offset"):
                assert getattr(a, k) == getattr(b, k), (trial, k)
        _eq(mine.osqp_plan.rho_vec, ref.osqp_plan.rho_vec, f"{trial} rho_vec")


def test_sparse_mpc_plan_rejects_bad_problems():
    from warpmpc_b200.jax_sqp import SparseMPCProblem

    rng = np.random.default_rng(0)
    one = _RandomStage(rng, 2, 0, 0, 1)
    with pytest.raises(ValueError):
        build_sparse_mpc_plan(SparseMPCProblem((one,)))  # needs a transition and a terminal stage
    with pytest.raises(ValueError):
        build_sparse_mpc_plan(SparseMPCProblem((_RandomStage(rng, 2, 3, 0, 1), _RandomStage(rng, 2, 0, 0, 1))))
    with pytest.raises(ValueError):
        build_sparse_mpc_plan(SparseMPCProblem((_RandomStage(rng, 2, 2, 0, 1), _RandomStage(rng, 2, 2, 0, 1))))
