"""Multi-process (one process per GPU) host logic for batched solves.

The QP instances are independent, so N GPUs run N independent batches: no
data-path collective.  What the ranks share is the plan (built from the same
representative instance on every rank, so every rank's tables are equal) and
the timing/aggregation steps: the step time is the maximum over ranks, the
converged-instance count the sum.  The process group carries only those
scalars (NCCL on GPUs, gloo for the CPU tests).
"""

from __future__ import annotations

import datetime
import hashlib
import os
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class RankEnv:
    world: int
    rank: int
    local: int


def rank_env() -> RankEnv:
    """World size, global and local rank from the torchrun environment."""
    return RankEnv(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def init(env: RankEnv, backend: str = "nccl", timeout_s: float = 120.0):
    """Join the process group (world > 1 only); returns the device for collectives."""
    import torch

    if backend == "nccl":
        torch.cuda.set_device(env.local)
        dev = torch.device("cuda", env.local)
    else:
        dev = torch.device("cpu")
    if env.world > 1:
        import torch.distributed as dist

        kw = {"device_id": dev} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dev


def finalize(env: RankEnv) -> None:
    if env.world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def barrier(env: RankEnv) -> None:
    if env.world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(value: float, env: RankEnv, device, op_name: str) -> float:
    if env.world == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, env: RankEnv, device) -> float:
    """Slowest rank's value (step times)."""
    return _reduce(value, env, device, "MAX")


def sum_over_ranks(value: float, env: RankEnv, device) -> float:
    """Whole-job total (converged instances)."""
    return _reduce(value, env, device, "SUM")


def instance_seed(base: int, rank: int) -> int:
    """Seed of a rank's own instances: every rank solves different problems."""
    return int(base) + int(rank)


def shard_bounds(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [start, stop) of ``total`` instances owned by ``rank``.

    Sizes differ by at most one; used when a fixed total batch is split
    (strong scaling) rather than each rank owning its own batch.
    """
    if world < 1 or not (0 <= rank < world) or total < 0:
        raise ValueError(f"bad shard request total={total} world={world} rank={rank}")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def plan_digest(plan) -> bytes:
    """Digest of everything in an OSQP plan that the kernels read."""
    h = hashlib.sha256()
    q = plan.qdldl_plan
    for arr in (q.p, q.lp, q.li, q.etree, plan.kkt_upper.indptr, plan.kkt_upper.indices, plan.kkt_upper.data,
                plan.p_to_kkt, plan.a_to_kkt, plan.rho_to_kkt, plan.rho_vec, plan.scaling_d, plan.scaling_e,
                plan.p_scale, plan.a_scale, plan.q_scale):
        a = np.ascontiguousarray(np.asarray(arr))
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    h.update(np.float64(plan.scaling_c).tobytes())
    return h.digest()


def check_plans_agree(plan, env: RankEnv, device) -> None:
    """Raise on every rank if any two ranks built different plans."""
    if env.world == 1:
        return
    import torch
    import torch.distributed as dist

    d = np.frombuffer(plan_digest(plan), dtype=np.uint8).astype(np.int64)
    mine = torch.as_tensor(d, device=device)
    lo, hi = mine.clone(), mine.clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX)
    if not torch.equal(lo, hi):
        raise RuntimeError(f"rank {env.rank}: the ranks built different plans")
