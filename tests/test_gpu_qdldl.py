"""Batched LDL^T factor/solve on the GPU vs the oracle (float32, same op order).

The kernels and the oracle both follow the reference's operation order with
separately rounded products and sums, so L, D, D^-1 and the solution agree
bit for bit; the float64 oracle gives the error against exact arithmetic.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import qdldl_ref
from warpmpc_b200 import problems
from warpmpc_b200.jax_qdldl import build_qdldl_plan, compile_qdldl_variant

pytestmark = pytest.mark.gpu


def _spd_pattern(n, density, seed):
    rng = np.random.default_rng(seed)
    a = sp.random(n, n, density=density, random_state=seed)
    a = a + a.T + sp.eye(n) * (n + 1.0)
    return sp.csc_matrix(a)


def _values(plan, batch, seed, quasi_definite=False):
    rng = np.random.default_rng(seed)
    base = np.asarray(plan.a_data, dtype=np.float64)
    cols = np.repeat(np.arange(plan.n), np.diff(plan.a_indptr))
    diag = plan.a_indices == cols
    vals = np.empty((plan.nnz_a, batch))
    vals[~diag] = base[~diag, None] * (1.0 + 0.25 * rng.standard_normal((int((~diag).sum()), batch)))
    vals[diag] = base[diag, None] * rng.uniform(0.75, 1.25, size=(int(diag.sum()), batch))
    return vals.astype(np.float32)


CASES = [
    ("example4", sp.csc_matrix([[4.0, 1.0, 0.0, 0.0], [1.0, 3.0, 0.5, 0.0], [0.0, 0.5, 2.0, 0.25], [0.0, 0.0, 0.25, 1.0]])),
    ("diag1", sp.csc_matrix(np.array([[2.0]]))),
    ("rand40", _spd_pattern(40, 0.08, 3)),
    ("rand200", _spd_pattern(200, 0.02, 4)),
]


@pytest.mark.parametrize("name,mat", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("batch", [1, 37, 300])
def test_factor_solve_bitexact(cuda_device, name, mat, batch):
    import torch

    plan = build_qdldl_plan(mat)
    comp = compile_qdldl_variant(plan, np.float32, backend="cuda", transpose_work=True)
    vals = _values(plan, batch, seed=batch)
    rhs = np.random.default_rng(7).standard_normal((plan.n, batch)).astype(np.float32)
    x, lx, d = comp.factor_and_solve(torch.from_numpy(vals), torch.from_numpy(rhs))
    lx_o, d_o, dinv_o = qdldl_ref.factor(plan, vals)
    x_o = qdldl_ref.solve(plan, lx_o, dinv_o, rhs)
    np.testing.assert_array_equal(lx.cpu().numpy(), lx_o)
    np.testing.assert_array_equal(d.cpu().numpy(), d_o)
    np.testing.assert_array_equal(x.cpu().numpy(), x_o)
    # error vs float64
    x64 = qdldl_ref.solve(plan, *[qdldl_ref.factor(plan, vals.astype(np.float64))[i] for i in (0, 2)], rhs.astype(np.float64))
    rel = np.max(np.abs(x.cpu().numpy() - x64)) / max(1.0, np.max(np.abs(x64)))
    assert rel < 1e-4


def test_kkt_factor_solve_quadrotor(cuda_device):
    import torch

    b = problems.make_batch(problems.QUADROTOR, 64, seed=3)
    plan = problems.make_plan(b)
    from oracle import osqp_ref

    kkt = osqp_ref.assemble_kkt_values(plan, b.p_values, b.a_values)  # (B, nnz) float32
    comp = compile_qdldl_variant(plan.qdldl_plan, np.float32, backend="cuda", transpose_work=True)
    vals = np.ascontiguousarray(kkt.T)
    rhs = np.random.default_rng(1).standard_normal((plan.qdldl_plan.n, 64)).astype(np.float32)
    x, lx, d = comp.factor_and_solve(torch.from_numpy(vals), torch.from_numpy(rhs))
    lx_o, d_o, dinv_o = qdldl_ref.factor(plan.qdldl_plan, vals)
    np.testing.assert_array_equal(lx.cpu().numpy(), lx_o)
    np.testing.assert_array_equal(x.cpu().numpy(), qdldl_ref.solve(plan.qdldl_plan, lx_o, dinv_o, rhs))


def test_shared_factor_broadcast(cuda_device):
    import torch

    plan = build_qdldl_plan(CASES[2][1])
    comp = compile_qdldl_variant(plan, np.float32, backend="cuda", transpose_work=True)
    vals = _values(plan, 1, seed=2)
    lx, d, dinv = comp.factor(torch.from_numpy(vals))
    rhs = np.random.default_rng(3).standard_normal((plan.n, 50)).astype(np.float32)
    x = comp.solve(lx, dinv, torch.from_numpy(rhs)).cpu().numpy()
    lx_o, d_o, dinv_o = qdldl_ref.factor(plan, vals)
    np.testing.assert_array_equal(x, qdldl_ref.solve(plan, lx_o, dinv_o, rhs))


def test_empty_batch_and_bad_shapes(cuda_device):
    import torch

    plan = build_qdldl_plan(CASES[0][1])
    comp = compile_qdldl_variant(plan, np.float32, backend="cuda", transpose_work=True)
    lx, d, dinv = comp.factor(torch.zeros((plan.nnz_a, 0)))
    assert lx.shape == (plan.nnz_l, 0)
    with pytest.raises(ValueError):
        comp.factor(torch.zeros((plan.nnz_a + 1, 3)))
    with pytest.raises(TypeError):
        comp.factor(torch.zeros((plan.nnz_a, 3), dtype=torch.float64))


@pytest.mark.parametrize("cls", [problems.SMALL, problems.QUADROTOR], ids=lambda c: c.name)
def test_tma_solve_many_tiles(cuda_device, monkeypatch, cls):
    """The TMA-fed solve (batch a multiple of 4, one factor per instance) over
    many tiles per CTA and a partial last tile: bit-identical to the
    one-lane-per-instance kernel (WMPC_SOLVE_STREAM_OFF=1) and to the oracle."""
    import torch

    from oracle import osqp_ref

    batch = 148 * 32 * 2 + 28  # more tiles than CTAs, last tile 28 lanes wide
    b = problems.make_batch(cls, batch, seed=8)
    plan = problems.make_plan(b)
    qp = plan.qdldl_plan
    comp = compile_qdldl_variant(qp, np.float32, backend="cuda", transpose_work=True)
    vals = np.ascontiguousarray(osqp_ref.assemble_kkt_values(plan, b.p_values, b.a_values).T)
    lx, d, dinv = comp.factor(torch.from_numpy(vals).cuda())
    rhs = torch.from_numpy(np.random.default_rng(4).standard_normal((qp.n, batch)).astype(np.float32)).cuda()
    x_tma = comp.solve(lx, dinv, rhs).cpu().numpy()
    monkeypatch.setenv("WMPC_SOLVE_STREAM_OFF", "1")
    x_one = comp.solve(lx, dinv, rhs).cpu().numpy()
    np.testing.assert_array_equal(x_tma, x_one)
    sl = slice(batch - 64, batch)  # the oracle on the last two tiles (the partial one included)
    want = qdldl_ref.solve(qp, lx.cpu().numpy()[:, sl], dinv.cpu().numpy()[:, sl], rhs.cpu().numpy()[:, sl])
    np.testing.assert_array_equal(x_tma[:, sl], want)
