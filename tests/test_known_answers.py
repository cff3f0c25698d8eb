"""Known answers from the reference's own tests, on the oracle and the planner.

tests/test_jax_osqp.py:17-152 and tests/test_jax_qdldl_segments.py:56-88 of
the reference.
"""

import itertools

import numpy as np
import scipy.sparse as sp

from oracle import osqp_ref
from warpmpc_b200.jax_osqp import OSQPSettings, build_osqp_plan
from warpmpc_b200.jax_qdldl.planning import (
    _make_adaptive_segments,
    _make_fixed_segments,
    _make_optimal_segments,
    _make_segments,
)


def test_vector_rho_known_answer():
    p = sp.csc_matrix([[4.0, 1.0], [1.0, 2.0]])
    a = sp.csc_matrix([[1.0, 1.0], [1.0, 0.0], [0.0, 1.0], [0.0, 0.0]])
    lower = np.array([0.2, -0.1, -1e30, -1e30])
    upper = np.array([0.2, 1e30, 0.4, 1e30])
    s = OSQPSettings(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=25, scaling=0, rho_is_vec=True)
    plan = build_osqp_plan(p, a, lower, upper, s, scaling_q=np.array([-1.0, -0.5]))
    np.testing.assert_allclose(plan.rho_vec, np.array([100.0, 0.1, 0.1, 1e-6]))
    np.testing.assert_array_equal(plan.constr_type, np.array([1, 0, 0, -1]))


def test_ill_conditioned_closed_form():
    p = sp.csc_matrix([[1e-4, 0.0], [0.0, 1e4]])
    a = sp.eye(2, format="csc")
    l, u, q = np.zeros(2), np.full(2, 10.0), np.array([-1.0, -1.0])
    plan = build_osqp_plan(p, a, l, u, OSQPSettings(max_iter=200, scaling=10, check_termination=0), scaling_q=q)
    assert not np.allclose(plan.p_scale, 1.0) and not np.allclose(plan.a_scale, 1.0)
    x, z, y, prim, dual, obj = osqp_ref.solve(plan, plan.p_upper.data[None], plan.a_matrix.data[None], q[None], l[None], u[None])
    np.testing.assert_allclose(x, [[10.0, 1e-4]], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(z, [[10.0, 1e-4]], rtol=1e-6, atol=1e-6)
    assert prim[0] < 1e-8 and dual[0] < 1e-8 and y[0, 0] > 0
    np.testing.assert_allclose(obj, [-9.99505], rtol=1e-8, atol=1e-8)


def test_factor_reuse_equals_solve_oracle():
    p = sp.csc_matrix([[4.0, 1.0], [1.0, 2.0]])
    a = sp.eye(2, format="csc")
    l, u = np.array([0.0, 0.0]), np.array([1.0, 1.0])
    q = np.array([[-1.0, -1.0], [-2.0, -0.5]])
    plan = build_osqp_plan(p, a, l, u, OSQPSettings(max_iter=80, scaling=5), scaling_q=q[0])
    pv, av = plan.p_upper.data[None], plan.a_matrix.data[None]
    lb, ub = np.broadcast_to(l, q.shape), np.broadcast_to(u, q.shape)
    lx, dinv = osqp_ref.factor(plan, pv, av)
    z0 = np.zeros((2, plan.m))
    a1 = osqp_ref.solve_with_factor_from_state(plan, lx, dinv, pv, av, q, lb, ub, np.zeros((2, 2)), z0, z0)
    a2 = osqp_ref.solve(plan, pv, av, q, lb, ub)
    for x1, x2 in zip(a1, a2):
        np.testing.assert_allclose(x1, x2, rtol=1e-10, atol=1e-10)


def _mask(counts):
    mask = np.zeros((len(counts), max(counts, default=0)), dtype=bool)
    for r, c in enumerate(counts):
        mask[r, :c] = True
    return mask


def _cost(counts, segs):
    return sum((int(c[-1]) + 1 - int(c[0])) * int(np.max(counts[int(c[0]) : int(c[-1]) + 1], initial=0)) for _, c in segs)


def test_segment_strategy_selector():
    counts = np.array([5, 1, 4, 1, 3])
    mask = _mask(counts.tolist())
    assert len(_make_segments(mask, segment_budget=3, segment_strategy="fixed")) == 3
    assert len(_make_segments(mask, segment_budget=3, segment_strategy="greedy")) <= 3
    assert len(_make_segments(mask, segment_budget=3, segment_strategy="optimal")) == 3
    assert [(s, c.tolist()) for s, c in _make_fixed_segments(mask, 3)] == [
        (s, c.tolist()) for s, c in _make_segments(mask, segment_budget=3, segment_strategy="fixed")
    ]


def test_optimal_crosses_zero_saving_splits():
    counts = np.array([100, 1, 1, 100])
    mask = _mask(counts.tolist())
    assert _cost(counts, _make_adaptive_segments(mask, 3)) == 400
    assert _cost(counts, _make_optimal_segments(mask, 3)) == 202


def test_optimal_matches_bruteforce():
    rng = np.random.default_rng(0)
    for n in range(1, 9):
        for _ in range(20):
            counts = rng.integers(0, 8, size=n)
            mask = _mask(counts.tolist())
            for k in range(1, n + 1):
                segs = _make_optimal_segments(mask, k)
                assert len(segs) == k
                best = min(
                    sum((b - a) * int(np.max(counts[a:b], initial=0)) for a, b in zip((0, *sp_), (*sp_, n)))
                    for sp_ in itertools.combinations(range(1, n), k - 1)
                )
                assert _cost(counts, segs) == best
