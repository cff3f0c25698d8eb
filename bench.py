#!/usr/bin/env python3
"""Throughput benchmark of the batched OSQP-ADMM hot path on B200.

Workload (one "step"): one warm-started batched solve of the linear quadrotor
MPC -- nx=12, nu=4, horizon 30 (KKT dimension 1356), batch 65536 per GPU,
float32, OSQP rho=0.1 (vector rho), sigma=1e-6, alpha=1.6, max_iter=25,
Ruiz scaling 10 -- every instance with its own A, B, Q, R, x0 (seeded
synthetic data; see warpmpc_b200/problems.py).  Steps form a closed MPC
loop: each step warm-starts from the previous step's (x, z, y).

The headline value is solves/s counting only instances whose primal and dual
residuals are both <= 1e-3, through the persistent fused kernel replayed from
a CUDA graph, inputs resident in HBM.  The same line carries the per-call
("plain") drop-in path, the end-to-end number through the public API with
pinned host buffers, the roofline of the dominant kernel, and the CPU
baseline (the oracle's C restatement on the host cores).

Multi-GPU: one process per GPU (torchrun); every rank solves its own 65536
instances (weak scaling, no collective in the data path); the step time is
the max over ranks of the CUDA-event time.

``--impl reference`` times the reference algorithm's CPU restatement on the
host cores instead (the reference's own JAX/Warp code cannot run here).
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "batched QP solves/s (res≤1e-3) persistent vs plain drop-in; fwd+bwd/fwd time"
RES_TOL = 1e-3


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--batch", type=int, default=65536, help="instances per GPU")
    ap.add_argument("--config", default="quadrotor", choices=("quadrotor", "small", "cartpole"))
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU-baseline sample duration")
    ap.add_argument("--no-grad", action="store_true", help="skip the forward+adjoint timing")
    ap.add_argument("--grad-batch", type=int, default=16384)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-size multi-class measurement")
    ap.add_argument("--mixed-batch", type=int, default=131072, help="instances over the four mixed classes")
    ap.add_argument("--no-line-search", action="store_true", help="skip the SQP line-search step timing")
    ap.add_argument("--no-assembly", action="store_true", help="skip the SQP QP assembly timing")
    ap.add_argument("--no-sqp", action="store_true", help="skip the SQP step timing")
    ap.add_argument("--no-sqp4", action="store_true", help="skip the nonlinear quadrotor SQP timing")
    ap.add_argument("--no-tune", action="store_true", help="library default schedules (no autotuning)")
    ap.add_argument("--sqp4-batch", type=int, default=262144, help="instances of the nonlinear SQP leg")
    return ap.parse_args()


def get_class(name):
    from warpmpc_b200 import problems

    return {"quadrotor": problems.QUADROTOR, "small": problems.SMALL, "cartpole": problems.CARTPOLE}[name]


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                if out:
                    self.samples.append([f.strip() for f in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        smax = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for name, val in zip(names, s[5:9]):
                if "Active" in val and "Not" not in val:
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(self.samples),
        }


def algorithmic_bytes_per_instance(plan, max_iter):
    """Roofline bytes of one persistent solve of one instance (float32).

    factor (factor_stream_kernel): KKT values read + L, D, D^-1 written; each
    ADMM iteration (admm_stream_kernel): L read twice (forward and backward
    sweep) + D^-1 read.  Index tables are shared by all instances and
    amortised to zero.  Returns (whole solve, factor, one iteration).
    """
    qp = plan.qdldl_plan
    factor = 4 * (plan.nnz_kkt + qp.nnz_l + 2 * qp.n)
    iteration = 4 * (2 * qp.nnz_l + qp.n)
    return factor + max_iter * iteration, factor, iteration


def measured_traffic(args, batch, form="plain", kernel="admm_stream_kernel"):
    """DRAM bytes of one launch of `kernel` at this batch, scaled from the ncu
    capture summarised in profiles/ (traffic grows with the instance count:
    every tile streams the same bytes); None when no capture covers the config
    and schedule form (plain or frontier) the launch ran."""
    import re

    name = f"{kernel}_{args.config}.md" if form == "plain" else f"{kernel}_{form}_{args.config}.md"
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            m = re.search(r"^traffic_bytes_per_instance:\s*(\d+)", f.read(), re.M)
    except OSError:
        return None
    return float(m.group(1)) * batch if m else None


def dist_setup(args):
    from warpmpc_b200 import multirank

    env = multirank.rank_env()
    if env.world > 1:
        multirank.init(env, "nccl", timeout_s=120.0)
    else:
        import torch

        if torch.cuda.is_available():
            torch.cuda.set_device(0)
    return env.world, env.rank, env.local


def _env(world):
    from warpmpc_b200 import multirank

    env = multirank.rank_env()
    assert env.world == world
    return env


def max_over_ranks(value: float, world: int) -> float:
    from warpmpc_b200 import multirank

    return multirank.max_over_ranks(value, _env(world), "cuda") if world > 1 else value


def barrier(world):
    from warpmpc_b200 import multirank

    if world > 1:
        multirank.barrier(_env(world))


def accuracy_vs_fp64(plan, p, a, q, l, u, warm, dev, cores):
    """The library's solve of a step's inputs (host arrays, float32) against a
    float64 run of the C restatement from the same inputs and warm start (the
    reference's JAX/Warp backends cannot run here): per instance the largest
    deviation of x, z, y relative to the float64 solution's largest entry."""
    import torch

    from oracle.cpu_baseline import CpuOSQP
    from warpmpc_b200.jax_osqp import compile_osqp

    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent", device=dev)
    t = lambda v: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).to(dev)  # noqa: E731
    got = comp.engine.solve(t(p), t(a), t(q), t(l), t(u), warm=tuple(t(w) for w in warm))
    got = [g.cpu().numpy().astype(np.float64) for g in got[:3]]
    f64 = lambda v: np.asarray(v, dtype=np.float64)  # noqa: E731
    ref = CpuOSQP(plan, np.float64).solve(f64(p), f64(a), f64(q), f64(l), f64(u), warm=tuple(f64(w) for w in warm),
                                         threads=cores)[:3]
    f32 = lambda v: np.asarray(v, dtype=np.float32)  # noqa: E731
    ref32 = CpuOSQP(plan, np.float32).solve(f32(p), f32(a), f32(q), f32(l), f32(u), warm=tuple(f32(w) for w in warm),
                                           threads=cores)[:3]
    out = {"instances": int(q.shape[0]), "iterations": int(plan.settings.max_iter),
           "rule": "per instance max|v - v64| / max|v64| for v in x, z, y (same inputs and warm start)",
           "fp32_restatement": {}}

    def rel(g, r):
        e = np.abs(g - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)
        return {"median": float(np.median(e)), "max": float(e.max())}

    for name, g, r, r32 in zip(("x", "z", "y"), got, ref, ref32):
        out[name] = rel(g, r)
        # the float32 C restatement's own error: what float32 arithmetic costs
        out["fp32_restatement"][name] = rel(r32.astype(np.float64), r)
    return out


def cpu_baseline(plan, batch_np, args, cls, seed, cores=None, dev=None):
    """Oracle C restatement on the host cores: one closed-loop warm-started
    step on a bounded sample (cold solve, state advanced by u0, timed warm solve).
    With ``dev``, also the library's error on the first 256 instances of that
    step against a float64 run of the restatement (``accuracy_vs_fp64``)."""
    from oracle.cpu_baseline import CpuOSQP
    from warpmpc_b200 import problems

    cpu = CpuOSQP(plan)
    cores = cores or os.cpu_count() or 1
    b = batch_np
    # calibrate the sample size to ~args.cpu_seconds of work
    probe = min(b.batch, max(64, 8 * cores))
    sl = slice(0, probe)
    t0 = time.perf_counter()
    cpu.solve(b.p_values[sl], b.a_values[sl], b.q[sl], b.l[sl], b.u[sl], threads=cores)
    per = (time.perf_counter() - t0) / probe
    sample = int(min(b.batch, max(probe, args.cpu_seconds / 2 / max(per, 1e-9))))
    sl = slice(0, sample)
    params = problems.draw_params(cls, b.batch, seed)
    loop = problems.ClosedLoop(cls, problems.MPCParams(cls, *[getattr(params, k)[sl] for k in
                                                            ("a", "b", "qd", "rd", "x0", "x_ref")]))
    lo, hi = b.l[sl].copy(), b.u[sl].copy()
    x, z, y, *_ = cpu.solve(b.p_values[sl], b.a_values[sl], b.q[sl], lo, hi, threads=cores)
    loop.advance_host(x, lo, hi)
    t0 = time.perf_counter()
    _, _, _, prim, dual, _ = cpu.solve(b.p_values[sl], b.a_values[sl], b.q[sl], lo, hi, warm=(x, z, y),
                                       threads=cores)
    dt = time.perf_counter() - t0
    ok = float(np.mean((prim <= RES_TOL) & (dual <= RES_TOL)))
    acc = None
    if dev is not None:
        k = slice(0, min(256, sample))
        acc = accuracy_vs_fp64(plan, b.p_values[k], b.a_values[k], b.q[k], lo[k], hi[k], (x[k], z[k], y[k]), dev,
                               cores)
    return {
        "accuracy_vs_fp64": acc,
        "value": sample * ok / dt,
        "unit": "solves/s",
        "cores": cpu.threads_used,
        "kind": "port",
        "sample": f"{sample} instances of the same workload, one closed-loop warm-started step (second of two), "
                  f"{plan.settings.max_iter} ADMM iterations, C restatement (oracle/c/osqp_cpu.c), "
                  f"{cpu.threads_used} threads; {ok:.3f} of the sample at res<=1e-3",
        "seconds": dt,
        "converged_fraction": ok,
    }


def run_reference(args):
    """--impl reference: the reference algorithm restated in C, on the host cores."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from warpmpc_b200 import problems

    cls = get_class(args.config)
    b = problems.make_batch(cls, args.batch, seed=1000)
    plan = problems.make_plan(b)
    from oracle.cpu_baseline import CpuOSQP

    cpu = CpuOSQP(plan)
    cores = os.cpu_count() or 1
    probe = min(b.batch, max(64, 8 * cores))
    t0 = time.perf_counter()
    cpu.solve(b.p_values[:probe], b.a_values[:probe], b.q[:probe], b.l[:probe], b.u[:probe], threads=cores)
    per = (time.perf_counter() - t0) / probe
    budget = 150.0 / max(1, args.steps + args.warmup)  # whole run within a few minutes
    sample = int(min(b.batch, max(probe, budget / max(per, 1e-9))))
    sl = slice(0, sample)
    params = problems.draw_params(cls, args.batch, 1000)
    loop = problems.ClosedLoop(cls, problems.MPCParams(cls, *[getattr(params, k)[sl] for k in
                                                            ("a", "b", "qd", "rd", "x0", "x_ref")]))
    lo, hi = b.l[sl].copy(), b.u[sl].copy()
    warm = None
    times, fracs = [], []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        x, z, y, prim, dual, _ = cpu.solve(b.p_values[sl], b.a_values[sl], b.q[sl], lo, hi, warm=warm,
                                           threads=cores)
        loop.advance_host(x, lo, hi)  # the instances' next states: the next step is a new QP
        dt = time.perf_counter() - t0
        warm = (x, z, y)
        if step >= args.warmup:
            times.append(dt)
            fracs.append(float(np.mean((prim <= RES_TOL) & (dual <= RES_TOL))))
    step_s = float(np.mean(times))
    value = sample * fracs[-1] / step_s
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config_dict(args, cls, plan, sample),
        "cpu_baseline": {
            "value": value, "unit": "solves/s", "cores": cpu.threads_used, "kind": "port",
            "sample": f"{sample} of {args.batch} instances per step (bounded), C restatement of the reference "
                      "algorithm (oracle/c/osqp_cpu.c); the reference's JAX/Warp backends cannot run on this "
                      "machine (jax and warp are not installed)",
        },
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "converged_fraction": fracs[-1],
    }
    print(json.dumps(line), flush=True)
    return 0


ADJOINT_ITERS = (15, 20, 25)  # adjoint ADMM iteration counts the gradient leg times


def gradient_timing(args, dev, world):
    """(forward + adjoint) / forward on nx=4, nu=1, N=50, 16384 instances.

    Forward: persistent solve (25 ADMM iterations) that keeps its factor;
    backward: the adjoint on that factor (cotangent of ||u0 - u_target||^2),
    timed at each adjoint iteration count of ADJOINT_ITERS, each with its
    accuracy against the FP64 finite-difference fixture.  `ratio` is the
    count equal to the forward's (25).
    """
    import torch

    from warpmpc_b200 import problems
    from warpmpc_b200.jax_osqp import compile_osqp

    cls = problems.CARTPOLE
    b = problems.make_batch(cls, args.grad_batch, seed=3000)
    plan = problems.make_plan(problems.make_batch(cls, 1, seed=3000))
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent", device=dev,
                        derivatives=True)
    eng = comp.engine
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    P, A, Q, L, U = (t(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u))
    ui = (cls.horizon + 1) * cls.nx
    u_target = torch.from_numpy(np.random.default_rng(7).standard_normal((b.batch, cls.nu)).astype(np.float32)).to(dev)

    def fwd():
        return eng.solve(P, A, Q, L, U, keep_factor=True)

    def bwd(out, iters):
        x, z, y = out[0], out[1], out[2]
        dx = torch.zeros_like(x)
        dx[:, ui : ui + cls.nu] = 2.0 * (x[:, ui : ui + cls.nu] - u_target)
        return eng.adjoint(eng.last_workspace, P, A, L, U, x, z, y, dx, None, max_iter=iters)

    fwd_iters = plan.settings.max_iter
    by_iters = {}
    fwd_runs = []
    for k in ADJOINT_ITERS:
        for _ in range(3):
            o = fwd()
            bwd(o, k)
        torch.cuda.synchronize()
        reps = 5
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        fwd_ms = bwd_ms = 0.0
        for _ in range(reps):
            e[0].record()
            o = fwd()
            e[1].record()
            bwd(o, k)
            e[2].record()
            torch.cuda.synchronize()
            fwd_ms += e[0].elapsed_time(e[1]) / reps
            bwd_ms += e[1].elapsed_time(e[2]) / reps
        fwd_ms = max_over_ranks(fwd_ms, world)
        bwd_ms = max_over_ranks(bwd_ms, world)
        fwd_runs.append(fwd_ms)
        by_iters[str(k)] = {"adjoint_ms": bwd_ms, "fwd_ms": fwd_ms, "ratio": (fwd_ms + bwd_ms) / fwd_ms,
                            "accuracy_vs_fd64": gradient_accuracy(k, dev)}
    main = by_iters.get(str(fwd_iters)) or by_iters[str(ADJOINT_ITERS[-1])]
    return {
        "accuracy_vs_fd64": main["accuracy_vs_fd64"],
        "workload": f"linear {cls.name} MPC nx={cls.nx} nu={cls.nu} N={cls.horizon}, {b.batch} instances/GPU, "
                    f"loss ||u0 - u_target||^2, forward {fwd_iters} ADMM iterations, adjoint {fwd_iters} "
                    f"(and {', '.join(str(k) for k in ADJOINT_ITERS)} in by_adjoint_iterations)",
        "fwd_ms": main["fwd_ms"],
        "adjoint_ms": main["adjoint_ms"],
        "ratio": main["ratio"],
        "by_adjoint_iterations": by_iters,
        "refactorizations_in_backward": 0,
    }


def gradient_accuracy(iters, dev):
    """The timed gradient's error at the same settings (forward 25 and adjoint
    `iters` ADMM iterations) on the 256 instances of the FP64 central-difference
    fixture tests/golden/adjoint_fd_cartpole.npz (converged float64 QP
    solves): per instance max |g - g_fd| / max(|g_fd|_inf, 1e-3) over diag Q,
    diag R and x0, split by whether the forward solve met residual <= 1e-3."""
    import torch

    from warpmpc_b200 import problems
    from warpmpc_b200.jax_osqp import compile_osqp

    g = np.load(os.path.join(ROOT, "tests", "golden", "adjoint_fd_cartpole.npz"))
    cls = problems.CARTPOLE
    n_inst = int(g["fd_grad"].shape[0])
    params = problems.draw_params(cls, n_inst, int(g["seed"]))
    plan = problems.make_plan(problems.make_batch(cls, 1, int(g["seed"])))
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent", device=dev,
                        derivatives=True, adjoint_iters=iters)
    leaves = {k: torch.from_numpy(getattr(params, k)).float().to(dev).requires_grad_(k in ("qd", "rd", "x0"))
              for k in ("a", "b", "qd", "rd", "x0", "x_ref")}
    p, a, q, l, u = (t.contiguous() for t in problems.qp_from_params(problems.MPCParams(cls, **leaves)))
    x, z, y, prim, dual, obj = comp.solve(p, a, q, l, u)
    ui = (cls.horizon + 1) * cls.nx
    ut = torch.from_numpy(np.random.default_rng(int(g["target_seed"])).standard_normal((n_inst, cls.nu))).float().to(dev)
    ((x[:, ui : ui + cls.nu] - ut) ** 2).sum().backward()
    grad = torch.cat([leaves["qd"].grad, leaves["rd"].grad, leaves["x0"].grad], 1).cpu().numpy().astype(np.float64)
    fd = g["fd_grad"]
    rel = np.max(np.abs(grad - fd), axis=1) / np.maximum(np.max(np.abs(fd), axis=1), 1e-3)
    conv = ((prim <= RES_TOL) & (dual <= RES_TOL)).cpu().numpy()
    out = {"instances": int(g["converged"].sum()), "forward_iterations": plan.settings.max_iter,
           "adjoint_iterations": iters}
    for name, sel in (("all", g["converged"]), ("forward_at_res_1e-3", g["converged"] & conv)):
        r = rel[sel]
        out[name] = {"count": int(sel.sum()), "median": float(np.median(r)), "p90": float(np.percentile(r, 90)),
                     "frac_le_1e-2": float(np.mean(r <= 1e-2))} if r.size else {"count": 0}
    return out


def line_search_timing(args, dev, world, plan, hbm_peak, peak_source):
    """The SQP line-search step after the QP solve (wmpc_sqp_line_search_step):
    bound violation, Armijo metric, filter selection over the default 4-step
    ladder and z + step d, one launch over args.batch instances of the bench
    class's QP sizes (z of size n, m constraint rows).  HBM-bound: reads z, d,
    q, l, g, u and the candidate evaluations, writes z_next."""
    import torch

    from warpmpc_b200.jax_sqp import FilterLineSearchSettings, line_search_step, make_step_lengths

    s = FilterLineSearchSettings()
    steps = torch.from_numpy(make_step_lengths(s).astype(np.float32)).to(dev)
    B, n, m, k = args.batch, plan.n, plan.m, int(steps.numel())
    g = torch.Generator(device=dev).manual_seed(5)
    r = lambda *shape: torch.randn(*shape, device=dev, generator=g)  # noqa: E731
    z, d, q, gv = r(B, n), r(B, n), r(B, n), r(B, m)
    lo, up = gv - r(B, m).abs(), gv + r(B, m).abs()
    bc, cc, cv = r(B), r(k, B), r(k, B).abs()

    def run():
        return line_search_step(settings=s, step_lengths=steps, z=z, direction=d, q=q, constraint_l=lo, g=gv,
                                constraint_u=up, baseline_cost=bc, candidate_costs=cc,
                                candidate_constraint_violations=cv)

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    from warpmpc_b200 import native

    reps = 20
    native.profile_begin()
    for _ in range(reps):
        run()
    torch.cuda.synchronize()
    # the library's own event pair brackets each launch on its stream
    ms_sum, launches, _ = native.profile_end()
    ms = max_over_ranks(ms_sum / max(launches, 1), world)
    per = 4 * (4 * n + 3 * m + 2 * k + 1) + 4 * 4 + 3
    gbs = B * per / (ms * 1e-3) / 1e9
    return {
        "workload": f"SQP line-search step after the QP solve: {B} instances/GPU, z of {n}, {m} constraint rows, "
                    f"{k}-step ladder, one launch (wmpc_sqp_line_search_step)",
        "ms": ms,
        "bytes_per_instance": per,
        "achieved_gbs": gbs,
        "peak_gbs": hbm_peak,
        "peak_source": peak_source,
        "frac": gbs / hbm_peak,
        "launches_timed": launches,
    }


def assembly_timing(args, dev, world, hbm_peak, peak_source):
    """Batched SQP QP assembly (wmpc_sqp_assemble) of the stage-wise quadrotor
    MPC (nx=12, nu=4, N=30: 31 stages) for args.batch instances: stage values
    evaluated and packed once outside the timed launches."""
    import torch

    from warpmpc_b200 import native, problems, sqp_problems
    from warpmpc_b200.jax_sqp import QPAssembler, build_sparse_mpc_plan

    cls = problems.QUADROTOR
    prob = sqp_problems.make_problem(cls)
    plan = build_sparse_mpc_plan(prob)
    B = args.batch
    data = sqp_problems.make_data(cls, B, seed=6)
    g = torch.Generator(device=dev).manual_seed(6)
    z = torch.randn(B, int(plan.z_offsets[-1]), device=dev, generator=g)
    p = torch.randn(B, cls.nx, device=dev, generator=g)
    asm = QPAssembler(plan, prob, device=dev)
    packed = asm.pack(sqp_problems.evaluate_stages(prob, data, z, p))
    del z, p
    for _ in range(3):
        asm.assemble(packed)
    torch.cuda.synchronize()
    reps = 10
    native.profile_begin()
    for _ in range(reps):
        asm.assemble(packed)
    torch.cuda.synchronize()
    ms_sum, launches, _ = native.profile_end()
    ms = max_over_ranks(ms_sum / max(launches, 1), world)
    t = asm.tables
    per = 4 * (asm.width + t["n"] + t["nnz_p"] + t["nnz_a"] + 5 * t["m"] + 1)
    gbs = B * per / (ms * 1e-3) / 1e9
    return {
        "workload": f"SQP QP assembly, stage-wise quadrotor MPC nx={cls.nx} nu={cls.nu} N={cls.horizon} "
                    f"({len(prob.stages)} stages), {B} instances/GPU, one launch (wmpc_sqp_assemble)",
        "ms": ms, "bytes_per_instance": per, "achieved_gbs": gbs, "peak_gbs": hbm_peak, "peak_source": peak_source,
        "frac": gbs / hbm_peak, "launches_timed": launches,
    }


def sqp_timing(args, dev, world):
    """One SQP step with the filter line search (SparseMPCSQP.line_search_step)
    of the stage-wise quadrotor MPC (nx=12, nu=4, N=30) for args.batch
    instances, replayed from a CUDA graph: model evaluation (torch, the
    caller's part), QP assembly, persistent OSQP solve (25 iterations), four
    candidate evaluations and the fused line-search step."""
    import torch

    from warpmpc_b200 import problems, sqp_problems
    from warpmpc_b200.jax_sqp import SparseMPCSQP, build_sparse_mpc_plan

    cls = problems.QUADROTOR
    prob = sqp_problems.make_problem(cls)
    plan = build_sparse_mpc_plan(prob)
    B = args.batch
    ev = sqp_problems.make_evaluator(prob, sqp_problems.make_data(cls, B, seed=8), dev)
    sqp = SparseMPCSQP(prob, plan, ev, device=dev)
    g = torch.Generator(device=dev).manual_seed(8)
    params = torch.rand(B, cls.nx, device=dev, generator=g) * 2 - 1
    z = torch.zeros(B, int(plan.z_offsets[-1]), device=dev)
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        for _ in range(2):
            sqp.line_search_step(z, params, None)
    torch.cuda.current_stream(dev).wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        out = sqp.line_search_step(z, params, None)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / reps, world)
    accepted = float(out.line_search.accepted.float().mean())
    del graph
    return {
        "workload": f"SQP step with filter line search, stage-wise quadrotor MPC nx={cls.nx} nu={cls.nu} "
                    f"N={cls.horizon}, {B} instances/GPU, 25 ADMM iterations, 4-step ladder, CUDA graph",
        "ms_per_step": ms, "instance_steps_per_s": B / (ms * 1e-3), "accepted_fraction": accepted,
    }


def nonlinear_sqp_timing(args, dev, world):
    """Nonlinear SQP: the rigid-body quadrotor (12 states, 4 motor thrusts,
    RK4 dt = 0.02, N = 40) over args.sqp4_batch instances per GPU, 5 SQP
    iterations with the filter line search, 25 ADMM iterations per QP (warm
    started from the previous QP), the whole solve replayed from a CUDA
    graph; then the same solve followed by the gradient of ||u0 - u_target||^2
    with respect to x0 and the cost weights through the last QP (adjoint on
    the kept factorization), also graphed.  Reports instance-solves/s, the
    residual of the dynamics after the iterations and (forward + adjoint) /
    forward."""
    import torch

    from warpmpc_b200 import multirank, quadrotor_sqp as qs

    B, horizon = args.sqp4_batch, 40
    data = qs.make_data(B, seed=multirank.instance_seed(7000, multirank.rank_env().rank))
    w = qs.QuadrotorSQP(horizon, data, dev, iterations=5, max_iter=25)
    u_target = torch.full((B, qs.NU), qs.U_HOVER, device=dev)
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        w.solve()
        zf, rf = w.solve(keep_factor=True)
        w.gradient(zf, rf, u_target)
    torch.cuda.current_stream(dev).wait_stream(s)
    torch.cuda.synchronize()
    # the warm-up's kept factorization (tens of GB at this batch) and cached
    # blocks go back to the device before the graphs allocate their own
    del zf, rf
    w.sqp.qp.engine.last_workspace = None
    gc.collect()
    torch.cuda.empty_cache()
    g_fwd, g_fb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_fwd):
        z_out, _ = w.solve()
    gc.collect()
    torch.cuda.empty_cache()
    with torch.cuda.graph(g_fb, pool=g_fwd.pool()):
        z_fb, r_fb = w.solve(keep_factor=True)
        grads = w.gradient(z_fb, r_fb, u_target)

    def timed(graph, reps):
        graph.replay()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / reps, world)

    reps = max(1, min(args.steps, 3))
    fwd_ms = timed(g_fwd, reps)
    fb_ms = timed(g_fb, reps)
    c, gv, lo, up = w.sqp.evaluate_nlp(z_out, w.x0)
    viol = (torch.clamp(lo - gv, min=0) + torch.clamp(gv - up, min=0)).abs().amax(dim=1)
    finite = bool(torch.isfinite(grads[0]).all() and torch.isfinite(grads[1]).all() and torch.isfinite(grads[2]).all())
    del g_fwd, g_fb
    return {
        "workload": f"nonlinear quadrotor MPC (12 states, 4 thrusts, RK4 dt=0.02) N={horizon}, {B} instances/GPU, "
                    "5 SQP iterations x 25 ADMM iterations, filter line search, one CUDA graph",
        "ms_per_solve": fwd_ms, "instance_solves_per_s": B / (fwd_ms * 1e-3),
        "kkt_dim": int(w.plan.osqp_plan.qdldl_plan.n), "nnz_l": int(w.plan.osqp_plan.qdldl_plan.nnz_l),
        "max_violation_median": float(viol.median()), "frac_violation_le_1e-3": float((viol <= 1e-3).float().mean()),
        "fwd_adjoint_ms": fb_ms, "fwd_bwd_over_fwd": fb_ms / fwd_ms, "gradients_finite": finite,
        "gradient_wrt": "x0 (12), Q diagonal (12), R diagonal (4)",
    }


def mixed_timing(args, dev, world):
    """Mixed-size batch: args.mixed_batch instances spread over four linear MPC
    classes (nx, nu, N) = (4, 2, 10), (4, 2, 40), (12, 4, 20), (12, 4, 30),
    one multi-class persistent launch per step (wmpc_osqp_solve_persistent),
    at most 50 ADMM iterations with early exit (an instance stops once its
    primal residual and iterate change are at most 1e-3; SOLVED from exact
    residuals), in a closed MPC loop (every step each instance applies its u0
    and the next QP starts from its new state, warm-started from the previous
    solution), the whole step replayed from a CUDA graph.  Also times the same
    loop with a fixed 50 iterations.  Value: instances at primal/dual residual
    <= 1e-3 per second."""
    import torch

    from warpmpc_b200 import multirank, problems
    from warpmpc_b200.jax_osqp import OSQPSettings, compile_osqp, solve_classes

    classes = problems.MIXED_CLASSES
    per = max(1, args.mixed_batch // len(classes))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    engines, data, schedules = [], [], {}
    for k, cls in enumerate(classes):
        settings = OSQPSettings(**{**problems.DEFAULT_SETTINGS, "max_iter": 50})
        plan = problems.make_plan(problems.make_batch(cls, 1, seed=4000 + k), settings)
        seed = multirank.instance_seed(4000 + 10 * k, multirank.rank_env().rank)
        b = problems.make_batch(cls, per, seed=seed)
        best, _ = tuned_schedule(args, plan, b, dev, max_instances=per)
        comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent", device=dev,
                            schedule=best)
        engines.append(comp.engine)
        data.append((cls, seed, b))
        schedules[cls.name] = best

    res = {}
    for label, check in (("early_exit", 1), ("fixed50", 0)):
        # every label starts the loop from the same initial states
        items, loops = [], []
        for eng, (cls, seed, b) in zip(engines, data):
            items.append([eng, t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u), None])
            loops.append(problems.ClosedLoop(cls, problems.draw_params(cls, per, seed), device=dev))
        outs0 = solve_classes([tuple(it) for it in items], check_termination=check)  # cold start
        warm = [tuple(o[k].clone() for k in range(3)) for o in outs0]
        for it, w, lp, o in zip(items, warm, loops, outs0):
            it[6] = w
            lp.advance(o[0], it[4], it[5])

        def step():
            outs = solve_classes([tuple(it) for it in items], check_termination=check)
            for it, o, lp in zip(items, outs, loops):
                for k in range(3):
                    it[6][k].copy_(o[k])
                lp.advance(o[0], it[4], it[5])
            return outs

        s = torch.cuda.Stream(dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(s):
            for _ in range(max(3, args.warmup)):
                step()
        torch.cuda.current_stream(dev).wait_stream(s)
        torch.cuda.synchronize()
        graph = None
        try:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                outs = step()
        except Exception as exc:  # report, do not hide
            print(f"[bench] mixed: CUDA graph capture failed, timing eager launches: {exc!r}", file=sys.stderr)
            graph = None
        run = graph.replay if graph is not None else step
        for _ in range(2):
            r = run()
            outs = r if graph is None else outs
        torch.cuda.synchronize()
        barrier(world)
        steps = max(1, min(args.steps, 5))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            r = run()
            outs = r if graph is None else outs
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
        ok = sum(int(((o[3] <= RES_TOL) & (o[4] <= RES_TOL)).sum().item()) for o in outs)
        total_ok = multirank.sum_over_ranks(ok, multirank.rank_env(), dev) if world > 1 else ok
        res[label] = {
            "value": total_ok / (ms * 1e-3),
            "ms_per_step": ms,
            "converged_fraction": ok / (per * len(classes)),
            "mean_iters": {cls.name: float(o[6].float().mean().item()) for cls, o in zip(classes, outs)},
            "graphed": graph is not None,
        }
        del graph
    return {
        "workload": f"{per * len(classes)} instances/GPU over 4 linear MPC classes "
                    "(4,2,10) (4,2,40) (12,4,20) (12,4,30), closed MPC loop (state advanced by u0 every step, "
                    "warm-started), <= 50 ADMM iterations, one persistent launch per step, CUDA graph",
        "unit": "solves/s",
        "schedule_per_class": schedules,
        **res,
    }


# schedule candidates the bench's tuner times for each problem (the library
# defaults first); every candidate must reproduce the first one's iterates
# schedules the bench's tuner times (all give the same bits; measured on the quadrotor pattern at 65,536
# instances: the library's 24-unit chunks 59.8 ms per ADMM launch against 62.9 ms with 16)
TUNE_CANDIDATES = ({}, {"frontier_copies": 1}, {"units": 16, "cols": 16, "rel": 12, "funits": 16},
                   {"units": 16, "cols": 16, "rel": 12, "funits": 16, "frontier_copies": 1})


def tuned_schedule(args, plan, batch_np, dev, max_instances=65536):
    """The fastest schedule of this pattern on this device (autotune_stream,
    timed on up to max_instances of the workload's instances, cached per
    pattern and device for the process), or {} with --no-tune."""
    if args.no_tune:
        return {}, None
    from warpmpc_b200.jax_osqp.autotune import autotune_stream

    sl = slice(0, min(batch_np.batch, max_instances))
    try:
        r = autotune_stream(plan, batch_np.p_values[sl], batch_np.a_values[sl], batch_np.q[sl], batch_np.l[sl],
                            batch_np.u[sl], candidates=TUNE_CANDIDATES, repeats=3, device=dev,
                            cache_path=os.path.join("/tmp", "wmpc_bench_tune.json"))
    except Exception as exc:  # report, do not hide: the defaults run instead
        print(f"[bench] schedule tuning failed, library defaults used: {exc!r}", file=sys.stderr)
        return {}, None
    return r.best, [[c, round(ms, 3)] for c, ms in r.timings_ms]


def config_dict(args, cls, plan, batch):
    return {
        "workload": f"linear {cls.name} MPC nx={cls.nx} nu={cls.nu} N={cls.horizon}, warm-started closed loop",
        "instances_per_gpu": batch,
        "kkt_dim": int(plan.qdldl_plan.n),
        "nnz_kkt": int(plan.nnz_kkt),
        "nnz_l": int(plan.qdldl_plan.nnz_l),
        "max_iter": int(plan.settings.max_iter),
        "parallelism": f"dp{args.gpus} (instances sharded, no collective in the data path)",
        "l2": "inputs larger than L2 (L factors alone exceed 126 MB)",
    }


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    from warpmpc_b200 import multirank, native, problems
    from warpmpc_b200.jax_osqp import compile_osqp

    world, rank, local = dist_setup(args)
    dev = torch.device("cuda", local)
    cls = get_class(args.config)
    seed = multirank.instance_seed(1000, rank)
    b = problems.make_batch(cls, args.batch, seed=seed)
    b0 = problems.make_batch(cls, 1, seed=1000)  # plan from the same instance 0 on every rank
    plan = problems.make_plan(b0)
    if world > 1:
        multirank.check_plans_agree(plan, multirank.rank_env(), dev)
    schedule, tune_timings = tuned_schedule(args, plan, b, dev)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent", device=dev,
                        schedule=schedule)
    plain = None if args.no_plain else compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True,
                                                    mode="plain", device=dev)
    eng = comp.engine
    B = b.batch
    to_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    P, A, Q, L, U = (to_dev(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u))
    f32 = dict(dtype=torch.float32, device=dev)
    out = [torch.zeros((B, plan.n), **f32), torch.zeros((B, plan.m), **f32), torch.zeros((B, plan.m), **f32),
           torch.empty(B, **f32), torch.empty(B, **f32), torch.empty(B, **f32),
           torch.empty(B, dtype=torch.int32, device=dev), torch.empty(B, dtype=torch.int32, device=dev)]
    warm = (out[0], out[1], out[2])
    # closed MPC loop: after every solve each instance applies its u0 and the
    # next step's QP starts from the instance's new state (l = u = -x0 rows)
    loop = problems.ClosedLoop(cls, problems.draw_params(cls, args.batch, seed), device=dev)

    def step():
        eng.solve(P, A, Q, L, U, warm=warm, out=out)
        loop.advance(out[0], L, U)

    # cold solve to seed the warm start, then warm-up steps
    eng.solve(P, A, Q, L, U, out=out)
    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()

    graph = None
    if not args.no_graph:
        try:
            s = torch.cuda.Stream(device=dev)
            s.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(s):
                step()
            torch.cuda.current_stream(dev).wait_stream(s)
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                step()
            torch.cuda.synchronize()
            for _ in range(2):
                graph.replay()
            torch.cuda.synchronize()
        except Exception as exc:  # report, do not hide
            print(f"[bench] CUDA graph capture failed, timing eager launches: {exc!r}", file=sys.stderr)
            graph = None
    run_step = graph.replay if graph is not None else step

    # ---- timed region: persistent path -------------------------------------------------
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches_before = native.lib().wmpc_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev0.record()
        for _ in range(args.steps):
            run_step()
        ev1.record()
        torch.cuda.synchronize()
    barrier(world)
    elapsed_ms = ev0.elapsed_time(ev1)
    step_ms = max_over_ranks(elapsed_ms / args.steps, world)
    prim = out[3].cpu().numpy()
    dual = out[4].cpu().numpy()
    ok_frac = float(np.mean((prim <= RES_TOL) & (dual <= RES_TOL)))
    total_ok = ok_frac * B
    if world > 1:
        total_ok = multirank.sum_over_ranks(total_ok, multirank.rank_env(), dev)
    value = total_ok / (step_ms * 1e-3)

    # launches per step (graph replays bypass the host launch counter: count one eager step)
    native.profile_begin()
    step()
    dom_ms, dom_n, launches_step = native.profile_end()
    torch.cuda.synchronize()
    # the schedule form, CTAs per SM and grid of the step's streaming launch, as the library ran it
    launch = native.stream_last_launch()
    form = launch["form"] or "plain"
    # dominant kernel (admm_stream_kernel) and the factorization kernel
    # (factor_stream_kernel) each timed alone over the timed-region workload
    # (eager, same inputs; the library's event pair around each launch, on its stream)
    native.profile_begin(native.PROFILE_DOMINANT)
    for _ in range(args.steps):
        step()
    dom_ms, dom_n, _ = native.profile_end()
    native.profile_begin(native.PROFILE_FACTOR)
    for _ in range(args.steps):
        step()
    fac_ms, fac_n, _ = native.profile_end()
    dom_ms_per_launch = dom_ms / max(dom_n, 1)
    fac_ms_per_launch = fac_ms / max(fac_n, 1)
    per_inst, fac_b, it_b = algorithmic_bytes_per_instance(plan, plan.settings.max_iter)
    admm_bytes = plan.settings.max_iter * it_b * B  # what admm_stream_kernel alone must move
    factor_bytes = fac_b * B                         # what factor_stream_kernel alone must move
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_source = "measured" if "hbm_gbs" in peaks else "fallback"
    achieved = admm_bytes / (dom_ms_per_launch * 1e-3) / 1e9
    fac_achieved = factor_bytes / (fac_ms_per_launch * 1e-3) / 1e9 if fac_n else None
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": measured_traffic(args, B, form), "kernel": "admm_stream_kernel", "schedule": form,
        "ctas_per_sm": launch["ctas_per_sm"], "kernel_ms": dom_ms_per_launch, "launches_timed": dom_n,
        "bytes_per_launch": admm_bytes, "tuned_schedule": schedule, "tune_timings_ms": tune_timings,
        "bytes_rule": f"{plan.settings.max_iter} iterations x 4 (2 nnz(L) + n) per instance",
        "peak_source": peak_source,
        "factor": {
            "kernel": "factor_stream_kernel", "kernel_ms": fac_ms_per_launch, "launches_timed": fac_n,
            "bytes_per_launch": factor_bytes, "bytes_rule": "4 (nnz(KKT) + nnz(L) + 2 n) per instance",
            "achieved": fac_achieved, "peak": peak, "unit": "GB/s",
            "frac": (fac_achieved / peak) if fac_achieved else None,
            "traffic": measured_traffic(args, B, "plain", "factor_stream_kernel"),
        },
    }

    # ---- plain per-call drop-in ------------------------------------------------------
    plain_res = None
    if plain is not None:
        # the same closed loop, continued from the persistent loop's current states
        pe = plain.engine
        pout = [t.clone() for t in out]
        pwarm = (pout[0], pout[1], pout[2])
        PL, PU = L.clone(), U.clone()
        ploop = problems.ClosedLoop(cls, problems.draw_params(cls, args.batch, seed), device=dev)
        ploop.x0.copy_(loop.x0)

        def pstep():
            pe.solve(P, A, Q, PL, PU, warm=pwarm, out=pout)
            ploop.advance(pout[0], PL, PU)

        pstep()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        psteps = max(1, min(args.steps, 5))
        e0.record()
        for _ in range(psteps):
            pstep()
        e1.record()
        torch.cuda.synchronize()
        pms = max_over_ranks(e0.elapsed_time(e1) / psteps, world)
        pfrac = float(np.mean((pout[3].cpu().numpy() <= RES_TOL) & (pout[4].cpu().numpy() <= RES_TOL)))
        # the per-call kernels of one plain step, each timed by the library's event pairs
        native.profile_begin(native.PROFILE_DOMINANT)
        pstep()
        s_ms, s_n, _ = native.profile_end()
        native.profile_begin(native.PROFILE_FACTOR)
        pstep()
        f_ms, f_n, _ = native.profile_end()
        qp = plan.qdldl_plan
        solve_bytes = 4 * (2 * qp.nnz_l + 3 * qp.n) * B
        solve_ms = s_ms / max(s_n, 1)
        fac_ms = f_ms / max(f_n, 1)
        plain_res = {"value": multirank.sum_over_ranks(pfrac * B, multirank.rank_env(), dev) / (pms * 1e-3),
                     "ms_per_step": pms, "converged_fraction": pfrac, "steps": psteps,
                     "solve_kernel": {"ms_per_launch": solve_ms, "launches_per_step": s_n,
                                      "bytes_per_launch": solve_bytes,
                                      "bytes_rule": "4 (2 nnz(L) + 3 n) per instance (L twice, D^-1, rhs in, x out)",
                                      "achieved_gbs": solve_bytes / (solve_ms * 1e-3) / 1e9,
                                      "frac": solve_bytes / (solve_ms * 1e-3) / 1e9 / roofline["peak"]},
                     "factor_kernel": {"ms_per_launch": fac_ms, "launches_per_step": f_n,
                                       "bytes_per_launch": fac_b * B, "bytes_rule": "4 (nnz(KKT) + nnz(L) + 2 n)",
                                       "achieved_gbs": fac_b * B / (fac_ms * 1e-3) / 1e9 if f_n else None,
                                       "frac": (fac_b * B / (fac_ms * 1e-3) / 1e9 / roofline["peak"]) if f_n else None}}

    # ---- end to end through the public API with pinned host buffers --------------------
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        hP, hA, hQ = (pin(v) for v in (b.p_values, b.a_values, b.q))
        # the loop continues from the device loop's current states (l, u rows and x0)
        hL, hU = L.cpu().pin_memory(), U.cpu().pin_memory()
        hx, hz, hy = (torch.empty(tuple(t.shape), dtype=torch.float32).pin_memory() for t in out[:3])
        hx.copy_(out[0].cpu()); hz.copy_(out[1].cpu()); hy.copy_(out[2].cpu())
        hres = [torch.empty(B, dtype=torch.float32).pin_memory() for _ in range(3)]
        h2d = sum(t.numel() * 4 for t in (hP, hA, hQ, hL, hU, hx, hz, hy))
        d2h = sum(t.numel() * 4 for t in (hx, hz, hy, *hres))
        hloop = problems.ClosedLoop(cls, problems.draw_params(cls, args.batch, seed))
        hloop.x0_np[:] = loop.x0.cpu().numpy()

        def e2e_step():
            # host in, host out: the engine copies slices in and out on two streams while it solves;
            # then the host applies u0 and writes the instances' next states into l and u
            # (each slice's instances advance as soon as its results are on the host,
            # while the later slices are still being solved)
            comp.engine.solve_host(hP, hA, hQ, hL, hU, warm=(hx, hz, hy), out=(hx, hz, hy, *hres),
                                   on_slice=lambda s0, s1: hloop.advance_host(hx.numpy(), hL.numpy(), hU.numpy(),
                                                                              rows=(s0, s1)))

        e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        esteps = max(1, min(args.steps, 5))
        e0.record()
        for _ in range(esteps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / esteps, world)
        efrac = float(np.mean((hres[0].numpy() <= RES_TOL) & (hres[1].numpy() <= RES_TOL)))
        e2e = {"value": multirank.sum_over_ranks(efrac * B, multirank.rank_env(), dev) / (ems * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}

    # the headline legs are done: release their device memory (graph pool, engines,
    # workspaces, inputs) so that the larger side legs (262,144 nonlinear SQP
    # instances) start from an empty device
    graphed = graph is not None
    del graph, run_step, step
    del comp, eng, plain, P, A, Q, L, U, out, warm, loop
    if plain_res is not None:
        del pe, pout, pwarm, PL, PU, ploop, pstep
    if e2e is not None:
        del e2e_step
    gc.collect()
    torch.cuda.empty_cache()

    # ---- forward + adjoint vs forward (cartpole-like class, loss on u0) ------------------
    def side_leg(name, fn):
        """A secondary measurement: its failure is reported in its field and on
        stderr, not allowed to take the headline line down with it.  Each leg's
        device memory is returned to the device before the next one."""
        try:
            return fn()
        except Exception as exc:  # report, do not hide
            print(f"[bench] {name} measurement failed: {exc!r}", file=sys.stderr)
            return {"error": repr(exc)[:300]}
        finally:
            gc.collect()
            torch.cuda.empty_cache()

    grad = None
    if not args.no_grad:
        grad = side_leg("gradient", lambda: gradient_timing(args, dev, world))
    mixed = None
    if not args.no_mixed:
        mixed = side_leg("mixed", lambda: mixed_timing(args, dev, world))
    line_search = None
    if not args.no_line_search:
        line_search = side_leg("line search", lambda: line_search_timing(args, dev, world, plan, roofline["peak"],
                                                                          roofline["peak_source"]))
    assembly = None
    if not args.no_assembly:
        assembly = side_leg("assembly", lambda: assembly_timing(args, dev, world, roofline["peak"],
                                                                roofline["peak_source"]))
    sqp = None
    if not args.no_sqp:
        sqp = side_leg("sqp step", lambda: sqp_timing(args, dev, world))

    sqp4 = None
    if not args.no_sqp4:
        sqp4 = side_leg("nonlinear sqp", lambda: nonlinear_sqp_timing(args, dev, world))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(plan, b, args, cls, seed, dev=dev)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config_dict(args, cls, plan, B),
            "converged_fraction": ok_frac,
            "graphed": graphed,
            "plain": plain_res,
            "persistent_over_plain": (value / plain_res["value"]) if plain_res and plain_res["value"] else None,
            "fwd_bwd_over_fwd": grad.get("ratio") if grad else None,
            "gradient": grad,
            "mixed": mixed,
            "line_search": line_search,
            "assembly": assembly,
            "sqp_step": sqp,
            "nonlinear_sqp": sqp4,
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "accuracy_vs_fp64": cpu.pop("accuracy_vs_fp64") if cpu else None,
            "clocks": clocks.summary(),
            "gpu_launches": int(launches_step * args.steps),
            "algorithmic_bytes": {"per_instance": per_inst, "factor": fac_b, "iteration": it_b},
        }
        print(json.dumps(line), flush=True)
    multirank.finalize(multirank.rank_env())
    return 0


if __name__ == "__main__":
    sys.exit(main())
