"""Autotuner host logic (no GPU): knob application and restoration, best
selection, rejection of unknown knobs."""

import os

import pytest

from warpmpc_b200.jax_osqp.autotune import KNOBS, apply, select_best


def test_apply_sets_and_restores_knobs(monkeypatch):
    monkeypatch.setenv("WMPC_STREAM_UNITS", "7")
    monkeypatch.delenv("WMPC_STREAM_CTAS", raising=False)
    with apply({"units": 24, "ctas": 1}):
        assert os.environ["WMPC_STREAM_UNITS"] == "24" and os.environ["WMPC_STREAM_CTAS"] == "1"
    assert os.environ["WMPC_STREAM_UNITS"] == "7" and "WMPC_STREAM_CTAS" not in os.environ
    with pytest.raises(ValueError):
        with apply({"warps": 3}):
            pass
    assert set(KNOBS) >= {"units", "cols", "rel", "funits", "offload", "lstages", "sstages", "ctas"}


def test_select_best_keeps_the_earlier_of_ties():
    a, b, c = {}, {"units": 12}, {"units": 24}
    assert select_best([(a, 3.0), (b, 2.0), (c, 2.0)]) is b
    with pytest.raises(ValueError):
        select_best([])
