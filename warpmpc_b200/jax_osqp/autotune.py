"""Autotuner for the persistent streaming solve of one pattern.

The streaming kernel's schedule has a few free choices that do not change
any result bit (every candidate runs the same arithmetic in the same order):
how many units, columns and releases a backward chunk holds, how many units a
forward chunk holds, which leaf work moves to the releaser warps, the ring
depths, the CTAs per SM and (as a candidate knob, not a default candidate)
the frontier-slot form.  Which choice is fastest depends on the pattern
and the device, so ``autotune_stream`` times a list of candidates on a
representative batch and returns the fastest, checking on the way that every
candidate's iterates equal the first one's.  Results are cached per pattern
digest and device name.

The knobs are the library's schedule settings, read from the environment
when a compiled problem is created (each problem keeps the values it was
created with), so tuning and ``apply`` set them in the environment of this
process around the creation; ``compile_osqp(..., schedule=best)`` does the
same for one problem.
"""

from __future__ import annotations

import contextlib
import json
import os
from dataclasses import dataclass, field

import numpy as np

KNOBS = {
    "units": "WMPC_STREAM_UNITS",
    "cols": "WMPC_STREAM_COLS",
    "rel": "WMPC_STREAM_REL",
    "funits": "WMPC_STREAM_FUNITS",
    "offload": "WMPC_STREAM_OFFLOAD",
    "lstages": "WMPC_STREAM_LSTAGES",
    "sstages": "WMPC_STREAM_SSTAGES",
    "ctas": "WMPC_STREAM_CTAS",
    # the frontier-slot form: 0 none, 1 the only schedule (a problem compiled
    # so refuses solves that check termination), 2 (the library default)
    # beside the plain one where it lets two CTAs share an SM
    "frontier": "WMPC_STREAM_FRONTIER",
    "frontier_lag": "WMPC_STREAM_FRONTIER_LAG",
    # most CTAs per SM a fixed-iteration launch may use (2 to 4; capped by
    # what is resident on an SM: shared memory and registers)
    "max_ctas": "WMPC_STREAM_MAX_CTAS",
    # frontier form: rows without L entries copied into their slots from a
    # per-chunk list instead of being swept as units
    "frontier_copies": "WMPC_STREAM_FRONTIER_COPIES",
}

DEFAULT_CANDIDATES = (
    {},  # the library defaults (24-unit chunks)
    {"units": 16, "cols": 16, "rel": 12, "funits": 16},
    {"units": 12, "cols": 12, "rel": 10, "funits": 12},
    {"units": 16, "cols": 16, "rel": 12, "funits": 16, "offload": 1},
    {"frontier_copies": 1},
    {"ctas": 1},
)


@dataclass
class TuneResult:
    best: dict
    timings_ms: list = field(default_factory=list)  # (candidate, ms) in candidate order
    cached: bool = False


@contextlib.contextmanager
def apply(knobs: dict):
    """Set the schedule knobs for the problems compiled inside the block."""
    unknown = set(knobs) - set(KNOBS)
    if unknown:
        raise ValueError(f"unknown schedule knobs {sorted(unknown)}")
    saved = {k: os.environ.get(v) for k, v in KNOBS.items()}
    try:
        for k, v in knobs.items():
            os.environ[KNOBS[k]] = str(int(v))
        yield
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(KNOBS[k], None)
            else:
                os.environ[KNOBS[k]] = v


def _cache_key(plan, device_name: str) -> str:
    from ..multirank import plan_digest

    return f"{plan_digest(plan).hex()}:{device_name}"


def select_best(timings):
    """The fastest candidate; ties keep the earlier one."""
    best, best_ms = None, float("inf")
    for cand, ms in timings:
        if ms < best_ms:
            best, best_ms = cand, ms
    if best is None:
        raise ValueError("no candidate was timed")
    return best


def autotune_stream(plan, p_values, a_values, q, l, u, *, candidates=DEFAULT_CANDIDATES, repeats: int = 3,
                    device=None, cache_path: str | None = None, timer=None) -> TuneResult:
    """Time each candidate's persistent solve of (p_values, a_values, q, l, u)
    and return the fastest.  ``timer(solve) -> ms`` overrides the CUDA-event
    timing (tests); with ``cache_path`` a previous result for this pattern and
    device is returned without timing, and new results are stored there."""
    import torch

    from .solver import compile_osqp

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    dev_name = torch.cuda.get_device_name(dev) if dev.type == "cuda" else str(dev)
    key = _cache_key(plan, dev_name)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as fh:
            cache = json.load(fh)
        if key in cache:
            return TuneResult(best=dict(cache[key]["best"]), timings_ms=cache[key]["timings_ms"], cached=True)

    def cuda_timer(solve):
        for _ in range(2):
            solve()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            solve()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / repeats

    timer = timer or cuda_timer
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)  # noqa: E731
    args = [t(v) for v in (p_values, a_values, q, l, u)]
    timings, first = [], None
    for cand in candidates:
        with apply(cand):
            comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent",
                                device=dev)
            out = comp.solve(*args)
            got = [o.cpu().numpy() for o in out[:3]]
            if first is None:
                first = got
            else:
                for g, f in zip(got, first):
                    if not np.array_equal(g, f):
                        raise RuntimeError(f"schedule candidate {cand} changed the iterates")
            timings.append((dict(cand), float(timer(lambda: comp.solve(*args)))))
    result = TuneResult(best=select_best(timings), timings_ms=[[c, ms] for c, ms in timings])
    if cache_path:
        cache[key] = {"best": result.best, "timings_ms": result.timings_ms}
        with open(cache_path, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)
    return result


__all__ = ["DEFAULT_CANDIDATES", "KNOBS", "TuneResult", "apply", "autotune_stream", "select_best"]

