"""Filter line search: the oracle pinned to the reference's own known answers,
and the host-side pieces of the CUDA mirror (no GPU needed).

Known answers: ``tests/test_jax_sqp.py`` 95-145 of the reference (step ladder,
first accepted candidate on the cost branch, the baseline-cost acceptance
variant falling back to the last step, the bound-violation definition).
"""

import ctypes

import numpy as np
import pytest

from oracle import line_search_ref as ref
from warpmpc_b200 import native
from warpmpc_b200.jax_sqp import FilterLineSearchSettings, make_step_lengths

DEFAULTS = dict(g_max=1e-1, g_min=1e-3, gamma_c=1e-3, armijo_factor=1e-4, constraint_scale=0.1,
                cost_accept_uses_trial_cost=True)


def test_oracle_known_answer_first_accepted_candidate():
    steps = ref.make_step_lengths(0.5, 0.1)
    np.testing.assert_allclose(steps, [1.0, 0.5, 0.25, 0.125])
    f = np.float32
    step, cost, viol, reason, acc, _ = ref.filter_line_search(
        DEFAULTS, steps, np.array([10.0], f), np.array([1e-4], f), np.array([-2.0], f),
        np.array([[10.5], [9.0], [8.0]], f), np.array([[1e-4], [1e-4], [1e-4]], f))
    assert float(step[0]) == pytest.approx(0.5)
    assert int(reason[0]) == ref.COST and bool(acc[0])
    assert float(cost[0]) == 9.0


def test_oracle_known_answer_baseline_cost_branch_falls_back():
    steps = ref.make_step_lengths(0.5, 0.5)
    f = np.float32
    s = dict(DEFAULTS, cost_accept_uses_trial_cost=False)
    step, cost, viol, reason, acc, _ = ref.filter_line_search(
        s, steps, np.array([10.0], f), np.array([1e-4], f), np.array([-2.0], f),
        np.array([[9.0], [8.0]], f), np.array([[1e-4], [1e-4]], f))
    assert float(step[0]) == pytest.approx(0.5)
    assert int(reason[0]) == ref.MAX_ITER and not bool(acc[0])


def test_oracle_known_answer_constraint_violation():
    v = ref.constraint_violation(np.array([[0.0, -1.0, 2.0]]), np.array([[-1.0, 0.0, 3.0]]),
                                 np.array([[2.0, 1.0, 2.5]]), 0.1)
    assert float(v[0]) == pytest.approx(0.1 * np.sqrt(1.0 ** 2 + 0.5 ** 2))


@pytest.mark.parametrize("decay,step_min", [(0.5, 0.1), (0.5, 0.5), (0.7, 0.01), (0.9, 1.0), (0.5, 2.0)])
def test_step_ladder_matches_oracle(decay, step_min):
    got = make_step_lengths(FilterLineSearchSettings(line_search_step_decay=decay, line_search_step_min=step_min))
    np.testing.assert_array_equal(got, ref.make_step_lengths(decay, step_min))


@pytest.mark.parametrize("decay,step_min", [(0.0, 0.1), (1.0, 0.1), (0.5, 0.0)])
def test_step_ladder_rejects_bad_settings(decay, step_min):
    with pytest.raises(ValueError):
        make_step_lengths(FilterLineSearchSettings(line_search_step_decay=decay, line_search_step_min=step_min))


def test_settings_struct_matches_header():
    # six 4-byte fields (wmpc_line_search_settings)
    assert ctypes.sizeof(native.LineSearchSettings) == 24
    fields = [f[0] for f in native.SqpStepBatch._fields_]
    assert fields[:5] == ["batch", "n", "m", "n_steps", "n_candidates"] and len(fields) == 24
