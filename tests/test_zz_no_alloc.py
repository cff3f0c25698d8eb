"""wmpc_solve_noalloc: the allocation-free solve, called through the C ABI.

It exists for callers that cannot allocate device memory while solving (a
real-time control loop kept out of the CUDA allocator, or a custom-call
handler that only receives buffers from its host framework): its work
vectors live in a fixed array inside the library instead of a caller
workspace.  Its results must equal wmpc_solve's (the same arithmetic, so bit
for bit) on consecutive calls, which also shows that the contents the array
keeps from the previous call do not leak into the next one.  This file is
collected last so that, run after the other tests, the array has already
been through other work on the device.
"""

import ctypes

import numpy as np
import pytest

from warpmpc_b200 import native, problems
from warpmpc_b200.jax_qdldl import compile_qdldl_variant

pytestmark = pytest.mark.gpu


def _noalloc(lib, handle, lx, dinv, bstride, rhs, out, batch):
    import torch

    return lib.wmpc_solve_noalloc(handle, lx.data_ptr(), dinv.data_ptr(), bstride, rhs.data_ptr(), out.data_ptr(),
                                  batch, native.current_stream_handle(torch.device("cuda", 0)))


def test_solve_noalloc_matches_solve(cuda_device):
    import torch

    from oracle import osqp_ref

    batch = 300
    b = problems.make_batch(problems.QUADROTOR, batch, seed=77)
    plan = problems.make_plan(b)
    qp = plan.qdldl_plan
    comp = compile_qdldl_variant(qp, np.float32, backend="cuda", transpose_work=True)
    kkt = np.ascontiguousarray(osqp_ref.assemble_kkt_values(plan, b.p_values, b.a_values).T)
    lx, d, dinv = comp.factor(torch.from_numpy(kkt).cuda())
    lib = native.lib()
    handle = comp.device_plan.handle
    rng = np.random.default_rng(5)
    for call in range(2):
        rhs = torch.from_numpy(rng.standard_normal((qp.n, batch)).astype(np.float32)).cuda()
        expected = comp.solve(lx, dinv, rhs)
        out = torch.full((qp.n, batch), float("nan"), device="cuda")
        native.check(_noalloc(lib, handle, lx, dinv, 1, rhs, out, batch))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), expected.cpu().numpy(), err_msg=f"call {call}")
    # a shared factor (batch stride 0), still through the same array
    rhs = torch.from_numpy(rng.standard_normal((qp.n, 7)).astype(np.float32)).cuda()
    lx1, dinv1 = lx[:, :1].contiguous(), dinv[:, :1].contiguous()
    out = torch.empty((qp.n, 7), device="cuda")
    native.check(_noalloc(lib, handle, lx1, dinv1, 0, rhs, out, 7))
    np.testing.assert_array_equal(out.cpu().numpy(), comp.solve(lx1, dinv1, rhs).cpu().numpy())


def test_solve_noalloc_rejects_oversized_requests(cuda_device):
    import torch

    b = problems.make_batch(problems.QUADROTOR, 1, seed=1)
    qp = problems.make_plan(b).qdldl_plan
    comp = compile_qdldl_variant(qp, np.float32, backend="cuda", transpose_work=True)
    lib = native.lib()
    too_many = 8 * 1024 * 1024 // qp.n + 1
    dummy = torch.empty(1, device="cuda")
    rc = lib.wmpc_solve_noalloc(comp.device_plan.handle, dummy.data_ptr(), dummy.data_ptr(), 0, dummy.data_ptr(),
                                dummy.data_ptr(), too_many, native.current_stream_handle(torch.device("cuda", 0)))
    assert rc == native.WMPC_ERR_WORKSPACE
    assert b"exceeds its fixed scratch" in lib.wmpc_last_error_string()
