"""The finite-difference gradient fixture of the differentiation workload
(tests/golden/adjoint_fd_cartpole.npz, made by make_adjoint_fd.py) against
the exact active-set derivative at the converged float64 solution (oracle),
chained to diag(Q), diag(R) and x0 by hand.  Pins the fixture the GPU
gradient tests compare with."""

import os

import numpy as np

from oracle import adjoint_ref
from oracle.cpu_baseline import CpuOSQP
from warpmpc_b200 import problems

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adjoint_fd_cartpole.npz")


def test_fd_fixture_matches_exact_active_set_derivative():
    g = np.load(GOLDEN)
    cls = problems.CARTPOLE
    params = problems.draw_params(cls, int(g["fd_grad"].shape[0]), int(g["seed"]))
    plan = problems.make_plan(problems.make_batch(cls, 1, int(g["seed"])))
    ut = np.random.default_rng(int(g["target_seed"])).standard_normal((params.qd.shape[0], cls.nu))
    idx = np.flatnonzero(g["converged"])[:12]
    sub = problems.MPCParams(cls, *[getattr(params, k)[idx] for k in ("a", "b", "qd", "rd", "x0", "x_ref")])
    p, a, q, l, u = problems.qp_from_params(sub)
    x, z, y, prim, dual, _ = CpuOSQP(plan, np.float64).solve(p, a, q, l, u, max_iter=int(g["iters"]))
    ui = (cls.horizon + 1) * cls.nx
    p_ids, _ = problems._pattern_with_ids(cls)
    import scipy.sparse as sp

    pu = sp.triu(p_ids, format="csc")
    pu.sum_duplicates(); pu.sort_indices()
    ids = np.asarray(pu.data, dtype=np.int64) - 1
    worst = 0.0
    for r, i in enumerate(idx):
        dx = np.zeros(plan.n)
        dx[ui : ui + cls.nu] = 2.0 * (x[r, ui : ui + cls.nu] - ut[i])
        dq, dl, du, dp, _ = adjoint_ref.active_set_adjoint(plan, p[r], a[r], l[r], u[r], x[r], z[r], y[r], dx,
                                                           np.zeros(plan.m))
        grad = np.zeros(2 * cls.nx + cls.nu)
        for k in range(cls.nx):
            # diag(Q)_k: every P entry drawn from it, and q = -(Q x_ref) on every stage's state k
            grad[k] = dp[ids == k].sum() - sub.x_ref[r, k] * dq[k : (cls.horizon + 1) * cls.nx : cls.nx].sum()
            grad[cls.nx + cls.nu + k] = -(dl[k] + du[k])  # l = u = -x0 on the first nx rows
        for k in range(cls.nu):
            grad[cls.nx + k] = dp[ids == cls.nx + k].sum()
        fd = g["fd_grad"][i]
        worst = max(worst, float(np.max(np.abs(grad - fd)) / max(1e-3, np.max(np.abs(fd)))))
    assert worst < 1e-5, worst
