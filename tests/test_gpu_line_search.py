"""Filter line search and the SQP line-search step on the GPU against the oracle.

The selection reads its inputs element by element: step, cost, violation,
reason, accepted and every candidate's acceptance equal the float32 oracle
bit for bit.  The fused step's two row sums (bound violation, q . d) are warp
reductions (order differs from NumPy's), so the baseline violation is checked
to 1e-5 relative; z_next = z + step * d is elementwise and bit-exact.
"""

import numpy as np
import pytest

from oracle import line_search_ref as ref
from warpmpc_b200.jax_sqp import (
    LINE_SEARCH_COST,
    LINE_SEARCH_MAX_ITER,
    FilterLineSearchSettings,
    constraint_violation,
    filter_line_search_from_evaluations,
    line_search_step,
    make_step_lengths,
)

pytestmark = pytest.mark.gpu


def _oracle_settings(s: FilterLineSearchSettings) -> dict:
    return dict(g_max=s.line_search_g_max, g_min=s.line_search_g_min, gamma_c=s.line_search_gamma_c,
                armijo_factor=s.line_search_armijo_factor, constraint_scale=s.line_search_constraint_scale,
                cost_accept_uses_trial_cost=s.line_search_cost_accept_uses_trial_cost)


def _np(t):
    return t.cpu().numpy()


def test_known_answers_through_cuda(cuda_device):
    s = FilterLineSearchSettings(line_search_step_min=0.1, line_search_step_decay=0.5)
    r = filter_line_search_from_evaluations(
        settings=s, step_lengths=make_step_lengths(s), baseline_cost=np.array([10.0]),
        baseline_constraint_violation=np.array([1e-4]), armijo_descent_metric=np.array([-2.0]),
        candidate_costs=np.array([[10.5], [9.0], [8.0]]), candidate_constraint_violations=np.array([[1e-4]] * 3))
    assert float(r.step_length[0]) == 0.5 and int(r.reason[0]) == LINE_SEARCH_COST and bool(r.accepted[0])
    s2 = FilterLineSearchSettings(line_search_step_min=0.5, line_search_step_decay=0.5,
                                  line_search_cost_accept_uses_trial_cost=False)
    r2 = filter_line_search_from_evaluations(
        settings=s2, step_lengths=make_step_lengths(s2), baseline_cost=np.array([10.0]),
        baseline_constraint_violation=np.array([1e-4]), armijo_descent_metric=np.array([-2.0]),
        candidate_costs=np.array([[9.0], [8.0]]), candidate_constraint_violations=np.array([[1e-4]] * 2))
    assert float(r2.step_length[0]) == 0.5 and int(r2.reason[0]) == LINE_SEARCH_MAX_ITER
    assert not bool(r2.accepted[0])
    v = constraint_violation(np.array([[0.0, -1.0, 2.0]]), np.array([[-1.0, 0.0, 3.0]]),
                             np.array([[2.0, 1.0, 2.5]]), 0.1)
    assert float(v[0]) == pytest.approx(0.1 * np.sqrt(1.25), rel=1e-6)


def _random_evaluations(rng, n_cand, batch):
    """Candidate costs / violations and baselines spread over every branch:
    violations above g_max, below g_min and in between, costs around the
    baseline on a coarse grid (no ties with the acceptance bounds)."""
    f = np.float32
    viol_levels = np.array([0.0, 5e-4, 2e-3, 0.05, 0.2, 1.0, np.nan], f)
    cv = viol_levels[rng.integers(0, viol_levels.size - 1, (n_cand, batch))]
    cv[rng.random((n_cand, batch)) < 0.01] = np.nan
    bc = (rng.integers(-64, 64, batch) / 8.0).astype(f)
    cc = (bc[None, :] + rng.integers(-24, 24, (n_cand, batch)) / 16.0 + 1.0 / 64).astype(f)
    cc[rng.random((n_cand, batch)) < 0.01] = np.inf
    bv = viol_levels[rng.integers(0, viol_levels.size - 1, batch)]
    am = ((rng.random(batch) - 0.7) * 4.0).astype(f)
    return cc, cv, bc, bv, am


@pytest.mark.parametrize("trial_cost", [True, False])
@pytest.mark.parametrize("n_cand", [1, 3, 4, 6])
def test_filter_selection_bitexact(cuda_device, trial_cost, n_cand):
    rng = np.random.default_rng(7 + n_cand)
    s = FilterLineSearchSettings(line_search_cost_accept_uses_trial_cost=trial_cost)
    steps = make_step_lengths(s)  # 4 steps: fewer, equal and more candidates than steps
    batch = 20000
    cc, cv, bc, bv, am = _random_evaluations(rng, n_cand, batch)
    got = filter_line_search_from_evaluations(
        settings=s, step_lengths=steps, baseline_cost=bc, baseline_constraint_violation=bv,
        armijo_descent_metric=am, candidate_costs=cc, candidate_constraint_violations=cv)
    want = ref.filter_line_search(_oracle_settings(s), steps.astype(np.float32), bc, bv, am, cc, cv)
    np.testing.assert_array_equal(_np(got.step_length), want[0])
    np.testing.assert_array_equal(_np(got.cost), want[1])
    np.testing.assert_array_equal(_np(got.constraint_violation), want[2])
    np.testing.assert_array_equal(_np(got.reason), want[3])
    np.testing.assert_array_equal(_np(got.accepted), want[4])
    np.testing.assert_array_equal(_np(got.candidate_acceptance), want[5])
    # every branch was selected somewhere (with the baseline cost on the left of the
    # Armijo test the cost branch can never accept: armijo < 0 on that branch)
    assert set(want[3].tolist()) == ({0, 1, 2, 3} if trial_cost else {0, 1, 3})


def test_constraint_violation_rows(cuda_device):
    rng = np.random.default_rng(3)
    for batch, m in ((1, 1), (257, 0), (1000, 37), (64, 1000)):
        g = rng.standard_normal((batch, m)).astype(np.float32)
        lo = (g + rng.standard_normal((batch, m))).astype(np.float32)
        up = (lo + np.abs(rng.standard_normal((batch, m)))).astype(np.float32)
        got = _np(constraint_violation(lo, g, up, 0.1))
        want = ref.constraint_violation(lo.astype(np.float64), g.astype(np.float64), up.astype(np.float64), 0.1)
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=0)


@pytest.mark.parametrize("n,m", [(61, 47), (64, 48)])  # element-wise and 16-byte row paths
def test_line_search_step_against_oracle(cuda_device, n, m):
    rng = np.random.default_rng(11)
    s = FilterLineSearchSettings()
    steps = make_step_lengths(s).astype(np.float32)
    batch, n_cand = 5000, 4
    f = np.float32
    z = rng.standard_normal((batch, n)).astype(f)
    d = rng.standard_normal((batch, n)).astype(f)
    q = rng.standard_normal((batch, n)).astype(f)
    g = rng.standard_normal((batch, m)).astype(f)
    scale = rng.choice(np.array([0.0, 1e-3, 1.0], f), size=(batch, 1))  # every violation regime
    lo = (g - np.abs(rng.standard_normal((batch, m))) + scale * rng.standard_normal((batch, m))).astype(f)
    up = (g + np.abs(rng.standard_normal((batch, m))) + scale * rng.standard_normal((batch, m))).astype(f)
    cc, cv, bc, _, _ = _random_evaluations(rng, n_cand, batch)
    d[7, 3] = np.inf  # a non-finite direction: is_finite false whatever the step
    got = line_search_step(settings=s, step_lengths=steps, z=z, direction=d, q=q, constraint_l=lo, g=g,
                           constraint_u=up, baseline_cost=bc, candidate_costs=cc, candidate_constraint_violations=cv)
    bviol = _np(got.baseline_constraint_violation)
    want_bviol = ref.constraint_violation(lo.astype(np.float64), g.astype(np.float64), up.astype(np.float64), 0.1)
    np.testing.assert_allclose(bviol, want_bviol, rtol=1e-5, atol=1e-30)
    # the selection, fed the GPU's baseline violation and the float64 Armijo metric
    am = np.sum(q.astype(np.float64) * d.astype(np.float64), axis=1).astype(f)
    want = ref.filter_line_search(_oracle_settings(s), steps, bc, bviol, am, cc, cv)
    ok = np.isfinite(am)
    np.testing.assert_array_equal(_np(got.line_search.step_length)[ok], want[0][ok])
    np.testing.assert_array_equal(_np(got.line_search.reason)[ok], want[3][ok])
    np.testing.assert_array_equal(_np(got.line_search.accepted)[ok], want[4][ok])
    step = _np(got.line_search.step_length)
    np.testing.assert_array_equal(_np(got.z_next), z + step[:, None] * d)
    fin = _np(got.is_finite)
    assert not fin[7] and fin.sum() == batch - 1


def test_empty_and_ragged_sizes(cuda_device):
    import torch

    s = FilterLineSearchSettings()
    steps = make_step_lengths(s)
    r = filter_line_search_from_evaluations(
        settings=s, step_lengths=steps, baseline_cost=np.zeros(0), baseline_constraint_violation=np.zeros(0),
        armijo_descent_metric=np.zeros(0), candidate_costs=np.zeros((4, 0)),
        candidate_constraint_violations=np.zeros((4, 0)))
    assert r.step_length.numel() == 0
    # no constraint rows: zero violation; the step still selects
    z = torch.ones((3, 5), device=cuda_device)
    got = line_search_step(settings=s, step_lengths=steps, z=z, direction=z, q=-z, constraint_l=np.zeros((3, 0)),
                           g=np.zeros((3, 0)), constraint_u=np.zeros((3, 0)), baseline_cost=np.ones(3),
                           candidate_costs=np.full((4, 3), 0.5), candidate_constraint_violations=np.zeros((4, 3)))
    assert np.all(_np(got.baseline_constraint_violation) == 0) and np.all(_np(got.line_search.step_length) == 1.0)
    with pytest.raises(ValueError):
        filter_line_search_from_evaluations(
            settings=s, step_lengths=np.zeros(0), baseline_cost=np.zeros(1), baseline_constraint_violation=np.zeros(1),
            armijo_descent_metric=np.zeros(1), candidate_costs=np.zeros((1, 1)),
            candidate_constraint_violations=np.zeros((1, 1)))
