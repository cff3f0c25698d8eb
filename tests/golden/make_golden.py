"""Generate the golden planner fixtures from the reference's own code.

Run where the reference tree exists, naming it in WARPMPC_REFERENCE_ROOT
(this script falls back to /root/reference, where the development container
mounts it):  WARPMPC_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py

The reference's NumPy/SciPy planners are imported through the oracle's
placeholder-module shim (oracle/ref_import.py).  The AMD permutation comes
from this project's AMD (the reference takes it from the absent `qdldl`
package); every array downstream of the permutation is the reference's.
Fixtures are small .npz files committed next to this script; the tests read
them and never need the reference at run time.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
os.environ.setdefault("WARPMPC_REFERENCE_ROOT", "/root/reference")

from oracle import ref_import  # noqa: E402
from warpmpc_b200 import problems  # noqa: E402
from warpmpc_b200.jax_qdldl.amd import amd_order  # noqa: E402

QDLDL_FIELDS = [
    "a_indptr", "a_indices", "a_data", "aperm_indptr", "aperm_indices", "perm_to_orig", "orig_to_perm", "p", "pinv",
    "etree", "lnz", "lp", "li", "diag_pos", "init_rows", "init_pos", "init_mask", "process_cols", "process_lidx",
    "process_offsets", "process_mask", "col_rows", "col_lidx", "col_mask",
]
OSQP_FIELDS = [
    "p_to_kkt", "p_diag_sigma", "a_to_kkt", "rho_to_kkt", "a_rows", "a_cols", "p_full_rows", "p_full_cols",
    "p_full_value_map", "rho_vec", "rho_inv_vec", "constr_type", "scaling_d", "scaling_dinv", "scaling_e",
    "scaling_einv", "p_scale", "a_scale", "q_scale", "y_scale", "y_unscale",
]


def _save_qdldl(name, ns, matrix, upper, perm):
    ref_import.PERMUTATION_PROVIDER = lambda _m: perm
    plan = ns.core.build_qdldl_plan(matrix, upper=upper)
    out = {f"plan_{f}": getattr(plan, f) for f in QDLDL_FIELDS}
    out["n"] = plan.n
    out["nnz_l"] = plan.nnz_l
    m = sp.csc_matrix(matrix)
    out["input_data"], out["input_indices"], out["input_indptr"] = m.data, m.indices, m.indptr
    out["input_shape"] = np.asarray(m.shape)
    out["upper"] = np.asarray(upper)
    levels = ns.core._make_solve_levels(plan.col_rows, plan.col_mask)
    flat, offsets = ns.warp_backend._pack_levels(levels)
    out["levels_flat"], out["levels_offsets"] = flat, offsets
    for th in (1, 2, 4):
        sched = ns.warp_backend._make_level_schedule(levels, offsets, serial_width_threshold=th)
        out[f"schedule_t{th}"] = np.asarray([[0 if k == "serial" else 1, a, b, c, d] for k, a, b, c, d in sched],
                                            dtype=np.int64).reshape(-1, 5)
    for mask_name in ("process_mask", "col_mask"):
        for strat in ("fixed", "greedy", "optimal"):
            for budget in (1, 3, 8, 64):
                st, cn, wd = ns.warp_backend._make_segment_arrays(getattr(plan, mask_name), segment_budget=budget,
                                                                  segment_strategy=strat)
                key = f"seg_{mask_name}_{strat}_{budget}"
                out[key + "_starts"], out[key + "_counts"], out[key + "_widths"] = st, cn, wd
    np.savez_compressed(os.path.join(HERE, f"qdldl_{name}.npz"), **out)
    return plan


def _save_osqp(name, ns, p, a, l, u, settings_kw, q=None):
    ref_import.PERMUTATION_PROVIDER = amd_order
    settings = ns.osqp_types.OSQPSettings(**settings_kw)
    plan = ns.solver.build_osqp_plan(p, a, l, u, settings, scaling_q=q, derivatives=True)
    out = {f"plan_{f}": getattr(plan, f) for f in OSQP_FIELDS}
    dp = plan.derivative_plan  # the reference's adjoint KKT plan (solver.py:413-571)
    for f in dp.__dataclass_fields__:
        v = getattr(dp, f)
        if isinstance(v, np.ndarray):
            out[f"dplan_{f}"] = v
        elif isinstance(v, (int, float)) and not isinstance(v, bool):
            out[f"dplan_{f}"] = np.asarray(v)
    out["dplan_adj_data"], out["dplan_adj_indices"], out["dplan_adj_indptr"] = (
        dp.adjoint_upper.data, dp.adjoint_upper.indices, dp.adjoint_upper.indptr)
    out["dplan_perm"], out["dplan_lp"], out["dplan_li"] = dp.qdldl_plan.p, dp.qdldl_plan.lp, dp.qdldl_plan.li
    out["scaling_c"] = plan.scaling_c
    out["scaling_cinv"] = plan.scaling_cinv
    out["kkt_data"], out["kkt_indices"], out["kkt_indptr"] = plan.kkt_upper.data, plan.kkt_upper.indices, plan.kkt_upper.indptr
    out["perm"] = plan.qdldl_plan.p
    out["kkt_lp"], out["kkt_li"] = plan.qdldl_plan.lp, plan.qdldl_plan.li
    pm, am = sp.csc_matrix(p), sp.csc_matrix(a)
    out["p_data"], out["p_indices"], out["p_indptr"], out["p_shape"] = pm.data, pm.indices, pm.indptr, np.asarray(pm.shape)
    out["a_data"], out["a_indices"], out["a_indptr"], out["a_shape"] = am.data, am.indices, am.indptr, np.asarray(am.shape)
    out["l"], out["u"] = np.asarray(l, dtype=float), np.asarray(u, dtype=float)
    out["q"] = np.asarray(q, dtype=float) if q is not None else np.zeros(0)
    out["settings"] = np.asarray([settings_kw.get(k, getattr(settings, k)) for k in ("rho", "sigma", "alpha", "max_iter", "scaling")], dtype=float)
    out["rho_is_vec"] = np.asarray(bool(settings.rho_is_vec))
    np.savez_compressed(os.path.join(HERE, f"osqp_{name}.npz"), **out)


def _save_sqp(name, cls):
    """The reference's sparse MPC plan (sparse_mpc.py:532-691) of a synthetic
    stage-wise problem (warpmpc_b200/sqp_problems.py stage descriptions)."""
    from warpmpc_b200 import sqp_problems

    ref_import.PERMUTATION_PROVIDER = amd_order
    sm = ref_import.load_sqp()
    prob = sqp_problems.make_problem(cls)
    plan = sm.build_sparse_mpc_plan(sm.SparseMPCProblem(stages=prob.stages))
    out = {}
    for k in ("stage_var_dims", "param_dims", "constraint_dims"):
        out[k] = np.asarray(getattr(plan, k))
    for k in ("z_offsets", "param_offsets", "constraint_offsets", "representative_l", "representative_u"):
        out[k] = getattr(plan, k)
    for k in ("p_pattern", "a_pattern"):
        out[k + "_indices"], out[k + "_indptr"] = getattr(plan, k).indices, getattr(plan, k).indptr
    for k in ("q_cols", "p_pos", "a_pos"):
        out["asm_" + k] = np.concatenate([getattr(a, k) for a in plan.assemblies])
        out["asm_" + k + "_counts"] = np.asarray([getattr(a, k).size for a in plan.assemblies])
    for k in ("z_offset", "next_z_offset", "param_offset", "constraint_offset"):
        out["asm_" + k] = np.asarray([getattr(a, k) for a in plan.assemblies])
    out.update({f"osqp_{f}": getattr(plan.osqp_plan, f) for f in OSQP_FIELDS})
    np.savez_compressed(os.path.join(HERE, f"sqp_plan_{name}.npz"), **out)


def main():
    ns = ref_import.load()
    rng = np.random.default_rng(2024)
    ex = sp.csc_matrix([[4.0, 1.0, 0.0, 0.0], [1.0, 3.0, 0.5, 0.0], [0.0, 0.5, 2.0, 0.25], [0.0, 0.0, 0.25, 1.0]])
    _save_qdldl("example4", ns, ex, False, amd_order(sp.triu(ex, format="csc")))
    for i, (n, dens) in enumerate([(30, 0.1), (60, 0.05)]):
        a = sp.random(n, n, density=dens, random_state=100 + i)
        a = sp.csc_matrix(a + a.T + sp.eye(n) * n)
        _save_qdldl(f"rand{n}_amd", ns, a, False, amd_order(sp.triu(a, format="csc")))
        _save_qdldl(f"rand{n}_perm", ns, a, False, rng.permutation(n).astype(np.int32))
    # the reference test problems (tests/test_jax_osqp.py:23-50, 98-105)
    _save_osqp("vector_rho", ns, sp.csc_matrix([[4.0, 1.0], [1.0, 2.0]]),
               sp.csc_matrix([[1.0, 1.0], [1.0, 0.0], [0.0, 1.0], [0.0, 0.0]]),
               np.array([0.2, -0.1, -1e30, -1e30]), np.array([0.2, 1e30, 0.4, 1e30]),
               dict(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=25, scaling=0, rho_is_vec=True),
               q=np.array([-1.0, -0.5]))
    _save_osqp("ill_conditioned", ns, sp.csc_matrix([[1e-4, 0.0], [0.0, 1e4]]), sp.eye(2, format="csc"),
               np.zeros(2), np.full(2, 10.0), dict(max_iter=200, scaling=10), q=np.array([-1.0, -1.0]))
    for cls in (problems.SMALL, problems.CARTPOLE):
        b = problems.make_batch(cls, 1, seed=7)
        _save_osqp(f"mpc_{cls.name}", ns, b.p_matrix0, b.a_matrix0, b.l[0].astype(float), b.u[0].astype(float),
                   dict(problems.DEFAULT_SETTINGS), q=b.q[0].astype(float))
    # the plans the bench solves: the quadrotor class from the headline
    # workload's instance 0 (seed 1000), and the two mixed-batch classes no
    # other fixture covers (instance 0 of their seeds 4000 + k)
    b = problems.make_batch(problems.QUADROTOR, 1, seed=1000)
    _save_osqp("mpc_quadrotor", ns, b.p_matrix0, b.a_matrix0, b.l[0].astype(float), b.u[0].astype(float),
               dict(problems.DEFAULT_SETTINGS), q=b.q[0].astype(float))
    for k, cls in enumerate(problems.MIXED_CLASSES):
        if cls.name in ("small-n40", "quad-n20"):
            b = problems.make_batch(cls, 1, seed=4000 + k)
            _save_osqp(f"mpc_{cls.name}", ns, b.p_matrix0, b.a_matrix0, b.l[0].astype(float), b.u[0].astype(float),
                       dict(problems.DEFAULT_SETTINGS, max_iter=50), q=b.q[0].astype(float))
    _save_sqp("small", problems.SMALL)
    _save_sqp("quadrotor_n5", problems.MPCClass("quadrotor-n5", 12, 4, 5, 10.0, 2.0, 1.0, "quadrotor"))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
