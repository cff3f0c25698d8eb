"""Bounded waits of the streaming ADMM kernel (failure detection).

Every handshake wait between the kernel's warps gives up after a time limit
(2 s by default); a launch whose waits gave up must still return, mark every
instance WMPC_STATUS_KERNEL_ABORT, and leave the context usable.  The test
makes the waits run out without faulting anything: it gives them a limit of
one microsecond (WMPC_STREAM_WAIT_LIMIT_NS), so the first wait that does not
succeed at once gives up.  The bulk copies already issued are still waited
for (with the 2 s limit) before the kernel returns.  A normal solve right
after must equal the oracle bit for bit.
"""

import numpy as np
import pytest

from oracle import osqp_ref
from warpmpc_b200 import native, problems
from warpmpc_b200.jax_osqp import compile_osqp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["plain", "frontier"])
def test_wait_timeout_aborts_cleanly(cuda_device, monkeypatch, form):
    import torch

    # the schedule form is fixed when the problem is created: 0 plain only, 1 frontier only
    monkeypatch.setenv("WMPC_STREAM_FRONTIER", "0" if form == "plain" else "1")
    b = problems.make_batch(problems.CARTPOLE, 96, seed=5)
    plan = problems.make_plan(b)
    comp = compile_osqp(plan, np.float32, qdldl_backend="cuda", transpose_work=True, mode="persistent",
                        device=cuda_device)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)  # noqa: E731
    args = [t(v) for v in (b.p_values, b.a_values, b.q, b.l, b.u)]
    monkeypatch.setenv("WMPC_STREAM_WAIT_LIMIT_NS", "1000")
    comp.engine.solve(*args)
    torch.cuda.synchronize()
    assert native.stream_last_launch()["form"] == form
    status = comp.engine.last_status.cpu().numpy()
    assert np.all(status & native.STATUS_KERNEL_ABORT), np.unique(status)
    monkeypatch.delenv("WMPC_STREAM_WAIT_LIMIT_NS")
    got = [o.cpu().numpy() for o in comp.engine.solve(*args)]
    status = comp.engine.last_status.cpu().numpy()
    assert not np.any(status & native.STATUS_KERNEL_ABORT)
    ref = osqp_ref.solve(plan, b.p_values, b.a_values, b.q, b.l, b.u)
    for name, g, r in zip(("x", "z", "y"), got[:3], ref[:3]):
        np.testing.assert_array_equal(g, r, err_msg=name)
