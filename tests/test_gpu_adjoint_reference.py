"""The reference's adjoint algorithm on the CUDA kernels (parity mode).

``ReferenceAdjoint`` runs the reference's augmented adjoint KKT (derivative
plan, eps-regularized factorization, 100 refinement steps against the
unperturbed matrix) with wmpc_factor / wmpc_solve / wmpc_sym_matvec in
float32; the oracle runs the same algorithm densely in float64
(``oracle/adjoint_ref.py``) on the same forward solution and cotangents.
"""

import numpy as np
import pytest

from oracle import adjoint_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_osqp import compile_osqp
from warpmpc_b200.jax_osqp.adjoint_reference import ReferenceAdjoint

pytestmark = pytest.mark.gpu


def test_reference_adjoint_matches_float64_restatement(cuda_device):
    import torch

    b = problems.make_batch(problems.SMALL, 8, seed=17)
    plan = problems.make_plan(b, derivatives=True)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()  # noqa: E731
    x, z, y, *_ = comp.solve(t(b.p_values), t(b.a_values), t(b.q), t(b.l), t(b.u))
    rng = np.random.default_rng(3)
    dx = rng.standard_normal((8, plan.n)).astype(np.float32)
    dy = rng.standard_normal((8, plan.m)).astype(np.float32)
    ra = ReferenceAdjoint(plan)
    state = ra.compute(t(b.p_values), t(b.a_values), t(b.l), t(b.u), x, y, t(dx), t(dy))
    dq, dl, du = (v.cpu().numpy() for v in ra.get_vec(state))
    dP, dA = (v.cpu().numpy() for v in ra.get_mat(x, y, state))
    xs, ys = x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)
    errs = []
    for i in range(8):
        want = adjoint_ref.adjoint(plan, b.p_values[i].astype(np.float64), b.a_values[i].astype(np.float64),
                                   b.l[i].astype(np.float64), b.u[i].astype(np.float64), xs[i], ys[i],
                                   dx[i].astype(np.float64), dy[i].astype(np.float64))
        for g, w in zip((dq[i], dl[i], du[i], dP[i], dA[i]), want):
            fin = np.isfinite(w)
            assert np.array_equal(fin, np.isfinite(g)), "non-finite entries differ"
            scale = max(1e-6, float(np.max(np.abs(w[fin])))) if fin.any() else 1.0
            errs.append(float(np.max(np.abs(g[fin] - w[fin]))) / scale if fin.any() else 0.0)
    errs = np.asarray(errs)
    print("relative max errors: median %.2e max %.2e" % (np.median(errs), errs.max()))
    # measured on B200: median 1.4e-7, max 1.3e-6 (float32 factor + refinement vs float64 dense)
    assert np.median(errs) < 1e-5 and errs.max() < 1e-4, errs
