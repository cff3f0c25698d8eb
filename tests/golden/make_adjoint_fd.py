"""Finite-difference gradients for the differentiation workload (fixture).

Workload: the cart-pole-like linear MPC class (nx=4, nu=1, N=50, |u| <= 10),
256 instances drawn with seed 3100, loss L = ||u0* - u_target||^2 per
instance (u_target ~ N(0, 1), seed 3101), u0* the first input of the
converged QP solution.  For every instance this script computes central
finite differences (step 1e-6) of L with respect to the instance's diag(Q)
(which enters P and q), diag(R) and x0 (which enters l = u on the first nx
constraint rows), on float64 solves of the oracle's C restatement run to
convergence (10000 ADMM iterations, the plan of instance 0).  Instances whose
float64 solve does not reach residuals <= 1e-9 are marked and excluded by the
tests.

Run:  python tests/golden/make_adjoint_fd.py   (writes adjoint_fd_cartpole.npz)
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.cpu_baseline import CpuOSQP  # noqa: E402
from warpmpc_b200 import problems  # noqa: E402

SEED, TARGET_SEED, BATCH, STEP, ITERS = 3100, 3101, 256, 1e-6, 10000


def u_target(batch=BATCH, nu=problems.CARTPOLE.nu):
    return np.random.default_rng(TARGET_SEED).standard_normal((batch, nu))


def main():
    cls = problems.CARTPOLE
    params = problems.draw_params(cls, BATCH, SEED)
    plan = problems.make_plan(problems.make_batch(cls, 1, SEED))
    cpu = CpuOSQP(plan, np.float64)
    ui = (cls.horizon + 1) * cls.nx
    ut = u_target()

    def solve(pr):
        p, a, q, l, u = problems.qp_from_params(pr)
        x, _, _, prim, dual, _ = cpu.solve(p, a, q, l, u, max_iter=ITERS)
        return np.sum((x[:, ui : ui + cls.nu] - ut) ** 2, axis=1), prim, dual

    t0 = time.time()
    loss, prim, dual = solve(params)
    names = [f"qd{k}" for k in range(cls.nx)] + [f"rd{k}" for k in range(cls.nu)] + [f"x0_{k}" for k in range(cls.nx)]
    grad = np.zeros((BATCH, len(names)))
    converged = (prim <= 1e-9) & (dual <= 1e-9)
    col = 0
    for field, width in (("qd", cls.nx), ("rd", cls.nu), ("x0", cls.nx)):
        for k in range(width):
            vals = []
            for sign in (1.0, -1.0):
                v = getattr(params, field).copy()
                v[:, k] += sign * STEP
                pr = problems.MPCParams(**{**params.__dict__, field: v})
                fl, fp, fd = solve(pr)
                converged &= (fp <= 1e-9) & (fd <= 1e-9)
                vals.append(fl)
            grad[:, col] = (vals[0] - vals[1]) / (2 * STEP)
            col += 1
    np.savez_compressed(os.path.join(HERE, "adjoint_fd_cartpole.npz"), seed=SEED, target_seed=TARGET_SEED, step=STEP,
                        iters=ITERS, names=np.asarray(names), fd_grad=grad, loss=loss, converged=converged,
                        prim=prim, dual=dual)
    print(f"{converged.sum()} of {BATCH} instances converged; {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
