"""Host planner vs the reference planners' own outputs (golden fixtures).

Fixtures were produced by the reference code itself
(tests/golden/make_golden.py); every table must match bit for bit.
"""

import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

from warpmpc_b200.jax_osqp import OSQPSettings, build_osqp_plan
from warpmpc_b200.jax_qdldl import build_qdldl_plan
from warpmpc_b200.jax_qdldl import planning as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
QD = sorted(glob.glob(os.path.join(GOLDEN, "qdldl_*.npz")))
OS = sorted(glob.glob(os.path.join(GOLDEN, "osqp_*.npz")))


def _eq(a, b, name):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.dtype == b.dtype, (name, a.dtype, b.dtype)
    assert a.shape == b.shape, (name, a.shape, b.shape)
    assert np.array_equal(a, b), name


@pytest.mark.parametrize("path", QD, ids=[os.path.basename(p) for p in QD])
def test_qdldl_plan_matches_reference(path):
    g = np.load(path)
    m = sp.csc_matrix((g["input_data"], g["input_indices"], g["input_indptr"]), shape=tuple(g["input_shape"]))
    plan = build_qdldl_plan(m, upper=bool(g["upper"]), perm=g["plan_p"])
    assert plan.n == int(g["n"]) and plan.nnz_l == int(g["nnz_l"])
    for k in g.files:
        if k.startswith("plan_"):
            _eq(getattr(plan, k[5:]), g[k], k)
    levels = P._make_solve_levels(plan.col_rows, plan.col_mask)
    flat, offsets = P._pack_levels(levels)
    _eq(flat, g["levels_flat"], "levels_flat")
    _eq(offsets, g["levels_offsets"], "levels_offsets")
    for th in (1, 2, 4):
        sched = P._make_level_schedule(levels, offsets, serial_width_threshold=th)
        arr = np.asarray([[0 if k == "serial" else 1, a, b, c, d] for k, a, b, c, d in sched], dtype=np.int64).reshape(-1, 5)
        _eq(arr, g[f"schedule_t{th}"], f"schedule_t{th}")
    for mask_name in ("process_mask", "col_mask"):
        for strat in ("fixed", "greedy", "optimal"):
            for budget in (1, 3, 8, 64):
                key = f"seg_{mask_name}_{strat}_{budget}"
                st, cn, wd = P._make_segment_arrays(getattr(plan, mask_name), segment_budget=budget, segment_strategy=strat)
                _eq(st, g[key + "_starts"], key)
                _eq(cn, g[key + "_counts"], key)
                _eq(wd, g[key + "_widths"], key)


@pytest.mark.parametrize("path", OS, ids=[os.path.basename(p) for p in OS])
def test_osqp_plan_matches_reference(path):
    g = np.load(path)
    p = sp.csc_matrix((g["p_data"], g["p_indices"], g["p_indptr"]), shape=tuple(g["p_shape"]))
    a = sp.csc_matrix((g["a_data"], g["a_indices"], g["a_indptr"]), shape=tuple(g["a_shape"]))
    rho, sigma, alpha, max_iter, scaling = g["settings"]
    settings = OSQPSettings(rho=rho, sigma=sigma, alpha=alpha, max_iter=int(max_iter), scaling=int(scaling),
                            rho_is_vec=bool(g["rho_is_vec"]))
    q = g["q"] if g["q"].size else None
    plan = build_osqp_plan(p, a, g["l"], g["u"], settings, scaling_q=q, perm=g["perm"], derivatives=True)
    for k in g.files:
        if k.startswith("plan_"):
            _eq(getattr(plan, k[5:]), g[k], k)
    # the reference-style adjoint KKT plan (solver.py:413-571)
    dp = plan.derivative_plan
    special = {"dplan_adj_data", "dplan_adj_indices", "dplan_adj_indptr", "dplan_perm", "dplan_lp", "dplan_li"}
    for k in g.files:
        if k.startswith("dplan_") and k not in special:
            _eq(np.asarray(getattr(dp, k[6:])), g[k], k)
    _eq(dp.adjoint_upper.data, g["dplan_adj_data"], "adjoint data")
    _eq(dp.adjoint_upper.indices, g["dplan_adj_indices"], "adjoint indices")
    _eq(dp.adjoint_upper.indptr, g["dplan_adj_indptr"], "adjoint indptr")
    _eq(dp.qdldl_plan.p, g["dplan_perm"], "adjoint perm")
    _eq(dp.qdldl_plan.lp, g["dplan_lp"], "adjoint lp")
    _eq(dp.qdldl_plan.li, g["dplan_li"], "adjoint li")
    assert plan.scaling_c == float(g["scaling_c"]) and plan.scaling_cinv == float(g["scaling_cinv"])
    _eq(plan.kkt_upper.data, g["kkt_data"], "kkt_data")
    _eq(plan.kkt_upper.indices, g["kkt_indices"], "kkt_indices")
    _eq(plan.kkt_upper.indptr, g["kkt_indptr"], "kkt_indptr")
    _eq(plan.qdldl_plan.lp, g["kkt_lp"], "kkt_lp")
    _eq(plan.qdldl_plan.li, g["kkt_li"], "kkt_li")


def test_live_reference_planners_random():
    """Direct comparison with the reference planners where the reference tree exists."""
    from oracle import ref_import

    if not ref_import.available():
        pytest.skip("reference checkout not present (fixtures cover this case)")
    ns = ref_import.load()
    from warpmpc_b200.jax_qdldl.amd import amd_order

    rng = np.random.default_rng(5)
    for trial in range(12):
        n = int(rng.integers(2, 50))
        m = sp.random(n, n, density=float(rng.uniform(0.03, 0.3)), random_state=int(rng.integers(1 << 30)))
        m = sp.csc_matrix(m + m.T + sp.eye(n) * n)
        perm = amd_order(sp.triu(m, format="csc")) if trial % 2 else rng.permutation(n).astype(np.int32)
        ref_import.PERMUTATION_PROVIDER = lambda _m, perm=perm: perm
        ref = ns.core.build_qdldl_plan(m)
        mine = build_qdldl_plan(m, perm=perm)
        for f in ref.__dataclass_fields__:
            x = getattr(ref, f)
            if isinstance(x, np.ndarray):
                _eq(getattr(mine, f), x, f)


def test_live_reference_derivative_plans_random():
    """The adjoint KKT plan against the reference's builder on random QPs with
    equality rows, one-sided and free rows (where the reference tree exists)."""
    from oracle import ref_import

    if not ref_import.available():
        pytest.skip("reference checkout not present (fixtures cover this case)")
    ns = ref_import.load()
    from warpmpc_b200.jax_osqp.derivative_plan import build_derivative_plan
    from warpmpc_b200.jax_qdldl.amd import amd_order

    ref_import.PERMUTATION_PROVIDER = amd_order
    rng = np.random.default_rng(9)
    for trial in range(8):
        n, m = int(rng.integers(2, 12)), int(rng.integers(1, 14))
        p = sp.random(n, n, density=0.3, random_state=int(rng.integers(1 << 30)))
        p = sp.triu(sp.csc_matrix(p @ p.T + sp.eye(n)), format="csc")
        a = sp.csc_matrix(sp.random(m, n, density=0.4, random_state=int(rng.integers(1 << 30))))
        a.sum_duplicates()
        a.sort_indices()
        kind = rng.integers(0, 4, m)  # 0 box, 1 equality, 2 lower only, 3 free
        l = np.where(kind == 3, -1e30, rng.standard_normal(m) - 1.0)
        u = np.where(kind == 2, 1e30, np.where(kind == 1, l, l + rng.uniform(0.1, 2.0, m)))
        u = np.where(kind == 3, 1e30, u)
        ref = ns.solver._build_derivative_plan(p, a, l, u)
        mine = build_derivative_plan(p, a, l, u)
        for f in ref.__dataclass_fields__:
            x = getattr(ref, f)
            if isinstance(x, np.ndarray):
                _eq(getattr(mine, f), x, f"trial {trial}: {f}")
            elif isinstance(x, (int, float)):
                assert getattr(mine, f) == x, (trial, f)
        _eq(mine.adjoint_upper.indices, ref.adjoint_upper.indices, "adjoint indices")
        _eq(mine.adjoint_upper.indptr, ref.adjoint_upper.indptr, "adjoint indptr")
        _eq(mine.adjoint_upper.data, ref.adjoint_upper.data, "adjoint data")
        _eq(mine.qdldl_plan.li, ref.qdldl_plan.li, "adjoint li")
