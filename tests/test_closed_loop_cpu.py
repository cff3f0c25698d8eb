"""The bench's closed MPC loop on the host: advancing the instances slice by
slice (as the host-buffer solve's per-slice callback does while the later
slices are still on the GPU) gives the states and bound rows of one
whole-batch advance."""

import numpy as np

from warpmpc_b200 import problems


def _loops(cls, batch, seed):
    params = problems.draw_params(cls, batch, seed)
    return problems.ClosedLoop(cls, params), problems.ClosedLoop(cls, problems.draw_params(cls, batch, seed))


def test_sliced_host_advance_equals_whole_batch():
    cls = problems.QUADROTOR
    batch = 1000
    whole, sliced = _loops(cls, batch, 5)
    b = problems.make_batch(cls, batch, seed=5)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((batch, b.q.shape[1])).astype(np.float32)
    l1, u1 = b.l.copy(), b.u.copy()
    l2, u2 = b.l.copy(), b.u.copy()
    whole.advance_host(x, l1, u1)
    for s0, s1 in ((0, 137), (137, 600), (600, 1000)):
        sliced.advance_host(x, l2, u2, rows=(s0, s1))
    np.testing.assert_allclose(sliced.x0_np, whole.x0_np, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(l2, l1, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(u2, u1, rtol=1e-6, atol=1e-7)
    # only the first nx bound rows move
    nx = cls.nx
    np.testing.assert_array_equal(l2[:, nx:], b.l[:, nx:])
    np.testing.assert_array_equal(u2[:, nx:], b.u[:, nx:])


def test_sliced_host_advance_touches_only_its_rows():
    cls = problems.SMALL
    batch = 64
    loop, _ = _loops(cls, batch, 9)
    b = problems.make_batch(cls, batch, seed=9)
    x = np.ones((batch, b.q.shape[1]), np.float32)
    x0_before = loop.x0_np.copy()
    l, u = b.l.copy(), b.u.copy()
    loop.advance_host(x, l, u, rows=(10, 20))
    np.testing.assert_array_equal(loop.x0_np[:10], x0_before[:10])
    np.testing.assert_array_equal(loop.x0_np[20:], x0_before[20:])
    assert not np.array_equal(loop.x0_np[10:20], x0_before[10:20])
    np.testing.assert_array_equal(l[:10], b.l[:10])
    np.testing.assert_array_equal(u[20:], b.u[20:])
