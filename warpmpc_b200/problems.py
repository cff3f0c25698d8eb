"""Seeded synthetic linear-MPC QP batches (fixed pattern, per-instance values).

Same QP layout as the reference's quadcopter MPC problem
(``benchmarks/problems/linear_mpc.py:109-132``): variables
``[x_0 .. x_N, u_0 .. u_{N-1}]``, cost ``blockdiag(I_N (x) Q, Q_N, I_N (x) R)``
with ``q = -blockdiag(Q..) x_ref``, equality rows ``x_{k+1} = A x_k + B u_k``
with ``x_0`` fixed by ``l = u = -x0`` on the first block, and a box on every
variable.  Every instance draws its own ``A, B, Q, R, x0, x_ref`` from
``np.random.default_rng(seed)``; the sparsity pattern is identical across
instances, so one plan (built from instance 0, as the reference builds its
scaling from representative values) serves the whole batch.

Configurations (the workload definitions of this project's benchmarks):

* ``small``  nx=4, nu=2, N=10: A = I + 0.1 G (G Gaussian, spectral radius of A
  rescaled to <= 1.02), B ~ N(0, 0.1), Q = diag U[1,10], R = diag U[0.1,1],
  Q_N = Q, |u| <= 1, |x| <= 5, x0 ~ U[-2,2];
* ``quadrotor`` nx=12, nu=4, N=30: A = I + 0.02 Ac, Ac ~ N(0,1) * 0.3 on a fixed
  block-sparse 3x3-block pattern, B ~ N(0, 0.5), Q/R as above, |u| <= 2,
  |x| <= 10, x0 ~ U[-1,1];
* ``cartpole`` nx=4, nu=1, N=50: as ``small`` with nu=1 and |u| <= 10.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from .jax_osqp.planning import build_osqp_plan
from .jax_osqp.types import OSQPSettings


@dataclass(frozen=True)
class MPCClass:
    name: str
    nx: int
    nu: int
    horizon: int
    x_max: float
    u_max: float
    x0_max: float
    kind: str = "small"  # "small" (dense A) or "quadrotor" (block-sparse A)


SMALL = MPCClass("small", 4, 2, 10, 5.0, 1.0, 2.0, "small")
QUADROTOR = MPCClass("quadrotor", 12, 4, 30, 10.0, 2.0, 1.0, "quadrotor")
CARTPOLE = MPCClass("cartpole", 4, 1, 50, 5.0, 10.0, 2.0, "small")
MIXED_CLASSES = (
    MPCClass("small-n10", 4, 2, 10, 5.0, 1.0, 2.0, "small"),
    MPCClass("small-n40", 4, 2, 40, 5.0, 1.0, 2.0, "small"),
    MPCClass("quad-n20", 12, 4, 20, 10.0, 2.0, 1.0, "quadrotor"),
    MPCClass("quad-n30", 12, 4, 30, 10.0, 2.0, 1.0, "quadrotor"),
)

DEFAULT_SETTINGS = dict(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=25, scaling=10, rho_is_vec=True)


def _quadrotor_mask(nx: int) -> np.ndarray:
    """Fixed block-sparse pattern of Ac (3x3 blocks: pos, att, vel, rate)."""
    nb = max(1, nx // 3)
    blocks = {(0, 2), (2, 1), (1, 3), (2, 2), (3, 3)}
    mask = np.zeros((nx, nx), dtype=bool)
    for bi in range(nb):
        for bj in range(nb):
            if (bi, bj) in blocks:
                mask[3 * bi : 3 * bi + 3, 3 * bj : 3 * bj + 3] = True
    return mask


def _draw_dynamics(cls: MPCClass, rng: np.random.Generator, batch: int):
    nx, nu = cls.nx, cls.nu
    if cls.kind == "quadrotor":
        mask = _quadrotor_mask(nx)
        ac = rng.standard_normal((batch, nx, nx)) * 0.3 * mask[None]
        a = np.eye(nx)[None] + 0.02 * ac
        b = rng.standard_normal((batch, nx, nu)) * 0.5
    else:
        g = rng.standard_normal((batch, nx, nx))
        a = np.eye(nx)[None] + 0.1 * g
        radius = np.max(np.abs(np.linalg.eigvals(a)), axis=1)
        shrink = np.minimum(1.0, 1.02 / radius)
        a = a * shrink[:, None, None]
        b = rng.standard_normal((batch, nx, nu)) * 0.1
    return a, b


def _pattern_with_ids(cls: MPCClass):
    """P and A of one symbolic instance whose values are source ids.

    Source ids index the flat per-instance vector
    ``[Q (nx), R (nu), A (nx*nx row-major), B (nx*nu row-major), -1, +1]``
    (1-based, so an explicit zero never appears).
    """
    nx, nu, N = cls.nx, cls.nu, cls.horizon
    q_ids = 1 + np.arange(nx)
    r_ids = 1 + nx + np.arange(nu)
    a_ids = 1 + nx + nu + np.arange(nx * nx).reshape(nx, nx)
    b_ids = 1 + nx + nu + nx * nx + np.arange(nx * nu).reshape(nx, nu)
    id_minus_one = 1 + nx + nu + nx * nx + nx * nu
    id_plus_one = id_minus_one + 1
    if cls.kind == "quadrotor":
        a_pat = (_quadrotor_mask(nx) | np.eye(nx, dtype=bool))
    else:
        a_pat = np.ones((nx, nx), dtype=bool)
    a_block = sp.csr_matrix(np.where(a_pat, a_ids, 0).astype(np.float64))
    b_block = sp.csr_matrix(b_ids.astype(np.float64))
    p_mat = sp.block_diag(
        [sp.kron(sp.eye(N), sp.diags(q_ids.astype(np.float64))), sp.diags(q_ids.astype(np.float64)),
         sp.kron(sp.eye(N), sp.diags(r_ids.astype(np.float64)))],
        format="csc",
    )
    ax = sp.kron(sp.eye(N + 1), sp.eye(nx) * id_minus_one) + sp.kron(sp.eye(N + 1, k=-1), a_block)
    bu = sp.kron(sp.vstack([sp.csc_matrix((1, N)), sp.eye(N)]), b_block)
    aeq = sp.hstack([ax, bu])
    nvar = (N + 1) * nx + N * nu
    aineq = sp.eye(nvar) * id_plus_one
    a_mat = sp.vstack([aeq, aineq], format="csc")
    for mat in (p_mat, a_mat):  # kron/bmat may store explicit zeros: they are not part of the pattern
        mat.sum_duplicates()
        mat.eliminate_zeros()
        mat.sort_indices()
    return p_mat, a_mat


@dataclass
class MPCBatch:
    cls: MPCClass
    p_matrix0: sp.csc_matrix   # instance 0 (true values)
    a_matrix0: sp.csc_matrix
    p_values: np.ndarray       # (B, nnz_p) in the plan's P-upper CSC order
    a_values: np.ndarray       # (B, nnz_a) in A's CSC order
    q: np.ndarray              # (B, n)
    l: np.ndarray              # (B, m)
    u: np.ndarray              # (B, m)
    x0: np.ndarray             # (B, nx)

    @property
    def batch(self) -> int:
        return int(self.q.shape[0])


@dataclass
class MPCParams:
    """The per-instance draws a batch is made of: dynamics ``A`` (B, nx, nx),
    ``B`` (B, nx, nu), cost diagonals ``qd`` (B, nx) and ``rd`` (B, nu), the
    initial state ``x0`` (B, nx) and the state reference ``x_ref`` (B, nx).
    Arrays are NumPy or torch (``qp_from_params`` is differentiable in torch)."""

    cls: MPCClass
    a: object
    b: object
    qd: object
    rd: object
    x0: object
    x_ref: object


def draw_params(cls: MPCClass, batch: int, seed: int = 0) -> MPCParams:
    """The seeded float64 draws of ``make_batch(cls, batch, seed)``, in its order."""
    rng = np.random.default_rng(seed)
    a, b = _draw_dynamics(cls, rng, batch)
    qd = rng.uniform(1.0, 10.0, size=(batch, cls.nx))
    rd = rng.uniform(0.1, 1.0, size=(batch, cls.nu))
    x0 = rng.uniform(-cls.x0_max, cls.x0_max, size=(batch, cls.nx))
    x_ref = rng.uniform(-0.5, 0.5, size=(batch, cls.nx))
    return MPCParams(cls, a, b, qd, rd, x0, x_ref)


def qp_from_params(params: MPCParams):
    """(p_values, a_values, q, l, u) of the instances' QPs, computed with the
    array module of ``params`` (NumPy float64, or torch so that gradients flow
    back to the draws: diag Q enters P and q, diag R enters P, x0 enters the
    first nx rows of l and u)."""
    cls = params.cls
    nx, nu, N = cls.nx, cls.nu, cls.horizon
    is_torch = not isinstance(params.qd, np.ndarray)
    if is_torch:
        import torch

        cat, tile = torch.cat, lambda t, reps: t.repeat(*reps)
        ones = lambda rows, val: torch.full((rows, 1), val, dtype=params.qd.dtype, device=params.qd.device)  # noqa: E731
        const = lambda arr: torch.as_tensor(arr, dtype=params.qd.dtype, device=params.qd.device)  # noqa: E731
        idx = lambda arr: torch.as_tensor(arr, dtype=torch.long, device=params.qd.device)  # noqa: E731
    else:
        cat, tile = (lambda xs, dim: np.concatenate(xs, axis=dim)), np.tile
        ones = lambda rows, val: np.full((rows, 1), val)  # noqa: E731
        const = idx = lambda arr: arr  # noqa: E731
    batch = params.qd.shape[0]
    sources = cat([params.qd, params.rd, params.a.reshape(batch, -1), params.b.reshape(batch, -1), ones(batch, -1.0),
                   ones(batch, 1.0)], 1)
    p_ids, a_ids = _pattern_with_ids(cls)
    p_upper = sp.triu(p_ids, format="csc")
    p_upper.sum_duplicates(); p_upper.sort_indices()
    p_values = sources[:, idx(np.asarray(p_upper.data, dtype=np.int64) - 1)]
    a_values = sources[:, idx(np.asarray(a_ids.data, dtype=np.int64) - 1)]
    nvar = (N + 1) * nx + N * nu
    m = (N + 1) * nx + nvar
    qx = -(params.qd * params.x_ref)
    q = cat([tile(qx, (1, N + 1)), const(np.zeros((batch, N * nu)))], 1)
    box_lo = np.concatenate([np.full((N + 1) * nx, -cls.x_max), np.full(N * nu, -cls.u_max)])
    lo_rest = np.concatenate([np.zeros(N * nx), box_lo])
    l = cat([-params.x0, const(np.broadcast_to(lo_rest, (batch, m - nx)).copy())], 1)
    hi_rest = np.concatenate([np.zeros(N * nx), -box_lo])
    u = cat([-params.x0, const(np.broadcast_to(hi_rest, (batch, m - nx)).copy())], 1)
    return p_values, a_values, q, l, u


class ClosedLoop:
    """Advances a batch's MPC instances one step in closed loop: every
    instance applies its first planned input, x0 <- A x0 + B u0 with its own
    (A, B), clipped inside the state box, and the new x0 is written into the
    first nx rows of l and u (l = u = -x0), so the next solve is a new QP.

    ``advance`` works on device tensors with torch operations (no host
    synchronisation: it can sit inside a captured CUDA graph);
    ``advance_host`` does the same on NumPy/host arrays."""

    def __init__(self, cls: MPCClass, params: MPCParams, device=None):
        self.cls = cls
        self.ui = (cls.horizon + 1) * cls.nx
        self.a_np = np.asarray(params.a, dtype=np.float32)
        self.b_np = np.asarray(params.b, dtype=np.float32)
        self.x0_np = np.asarray(params.x0, dtype=np.float32).copy()
        self.bound = np.float32(0.999 * cls.x_max)
        if device is not None:
            import torch

            self.a = torch.from_numpy(self.a_np).to(device)
            self.b = torch.from_numpy(self.b_np).to(device)
            self.x0 = torch.from_numpy(self.x0_np).to(device)

    def advance(self, x, l, u):
        """x: (B, n) solution on the device; l, u: (B, m) device tensors updated in place."""
        import torch

        nx, nu = self.cls.nx, self.cls.nu
        u0 = x[:, self.ui : self.ui + nu]
        nxt = torch.bmm(self.a, self.x0[:, :, None])[:, :, 0] + torch.bmm(self.b, u0[:, :, None])[:, :, 0]
        self.x0.copy_(nxt.clamp_(-float(self.bound), float(self.bound)))
        l[:, :nx] = -self.x0
        u[:, :nx] = -self.x0

    def advance_host(self, x, l, u, rows=None):
        """Host version of ``advance`` on NumPy arrays or host tensors (updated
        in place): the same torch operations on CPU (batched matrix products
        on the host's threads, through zero-copy views).  ``rows=(s0, s1)``
        advances only instances s0..s1-1 (x, l, u are still whole-batch arrays)."""
        import torch

        nx, nu = self.cls.nx, self.cls.nu
        s0, s1 = (0, self.x0_np.shape[0]) if rows is None else rows
        xt = torch.from_numpy(np.asarray(x, dtype=np.float32))[s0:s1]
        a, b, x0 = (torch.from_numpy(v)[s0:s1] for v in (self.a_np, self.b_np, self.x0_np))
        u0 = xt[:, self.ui : self.ui + nu]
        nxt = torch.bmm(a, x0[:, :, None])[:, :, 0] + torch.bmm(b, u0[:, :, None])[:, :, 0]
        x0.copy_(nxt.clamp_(-float(self.bound), float(self.bound)))
        for t in (l, u):
            torch.from_numpy(np.asarray(t))[s0:s1, :nx] = -x0


def make_batch(cls: MPCClass, batch: int, seed: int = 0, dtype=np.float32) -> MPCBatch:
    """Seeded batch of ``batch`` instances of class ``cls``."""
    params = draw_params(cls, batch, seed)
    p_values, a_values, q, l, u = qp_from_params(params)
    p_ids, a_ids = _pattern_with_ids(cls)
    p_upper = sp.triu(p_ids, format="csc")
    p_upper.sum_duplicates(); p_upper.sort_indices()
    p0 = sp.csc_matrix((p_values[0], p_upper.indices, p_upper.indptr), shape=p_upper.shape)
    a0 = sp.csc_matrix((a_values[0], a_ids.indices, a_ids.indptr), shape=a_ids.shape)
    return MPCBatch(
        cls=cls, p_matrix0=p0, a_matrix0=a0,
        p_values=p_values.astype(dtype), a_values=a_values.astype(dtype),
        q=q.astype(dtype), l=l.astype(dtype), u=u.astype(dtype), x0=params.x0.astype(dtype),
    )


def make_plan(batch: MPCBatch, settings: OSQPSettings | None = None, derivatives: bool = False, perm=None):
    """Plan from instance 0 (scaling and rho classification), like the reference."""
    settings = OSQPSettings(**DEFAULT_SETTINGS) if settings is None else settings
    return build_osqp_plan(
        batch.p_matrix0, batch.a_matrix0, batch.l[0].astype(np.float64), batch.u[0].astype(np.float64), settings,
        derivatives=derivatives, scaling_q=batch.q[0].astype(np.float64), perm=perm,
    )
