"""Seeded synthetic stage-wise MPC problems for the SQP QP assembly.

The reference builds its SQP problems from CasADi stage functions (absent
here); these are hand-written stage descriptions of the same shape, with
analytic derivatives, for tests and benchmarks of the assembly path.

Stage k < N: ``z_k = [x_k, u_k]`` (nx + nu), next input ``z_{k+1}`` (the
terminal stage's ``z_N = x_N``).  Cost ``0.5 (x' Q x + u' R u)`` (diagonal
Q, R per instance), constraints: dynamics ``x_{k+1} - A x_k - B u_k = 0``
(nx equality rows) and the input box ``-u_max <= u_k <= u_max`` (nu rows);
stage 0 also pins ``x_0 = p`` (nx equality rows, p = the parameters).  The
terminal stage costs ``0.5 x' Q x`` and has no constraints.  A and B come
from the ``problems`` module's class generators (per instance).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import problems
from .jax_sqp.assembly import SparseMPCProblem


@dataclass(frozen=True)
class LinearStage:
    """One stage's fixed local sparsity (the attributes the planner reads)."""

    k: int
    nx: int
    nu: int
    terminal: bool
    first: bool
    next_terminal: bool
    u_max: float

    @property
    def has_next(self):
        return not self.terminal

    @property
    def z_dim(self):
        return self.nx if self.terminal else self.nx + self.nu

    @property
    def next_z_dim(self):
        if self.terminal:
            return 0
        return self.nx if self.next_terminal else self.nx + self.nu

    @property
    def param_dim(self):
        return self.nx if self.first else 0

    @property
    def constraint_dim(self):
        if self.terminal:
            return 0
        return (self.nx if self.first else 0) + self.nx + self.nu

    @property
    def grad_cols(self):
        return np.arange(self.z_dim, dtype=np.int32)

    @property
    def hess_rows(self):
        return np.arange(self.z_dim, dtype=np.int32)

    @property
    def hess_cols(self):
        return np.arange(self.z_dim, dtype=np.int32)

    def _jac_pattern(self):
        """(rows, cols) of the constraint Jacobian, in a fixed order."""
        nx, nu = self.nx, self.nu
        rows, cols = [], []
        r0 = 0
        if self.first:
            rows += list(range(nx))
            cols += list(range(nx))
            r0 = nx
        for r in range(nx):  # dynamics row r: -A[r, :], -B[r, :], +1 on x_{k+1, r}
            rows += [r0 + r] * (nx + nu + 1)
            cols += list(range(nx + nu)) + [nx + nu + r]
        for j in range(nu):
            rows.append(r0 + nx + j)
            cols.append(nx + j)
        return np.asarray(rows, dtype=np.int32), np.asarray(cols, dtype=np.int32)

    @property
    def jac_rows(self):
        return self._jac_pattern()[0] if not self.terminal else np.zeros(0, np.int32)

    @property
    def jac_cols(self):
        return self._jac_pattern()[1] if not self.terminal else np.zeros(0, np.int32)

    def value_function(self, z, *rest):
        """(cost, g, lower, upper) of one instance with identity weights and
        dynamics (the planner only reads the bounds' types)."""
        p = rest[-1]
        cost = 0.5 * float(np.dot(z, z))
        if self.terminal:
            return cost, np.zeros(0), np.zeros(0), np.zeros(0)
        zn = rest[0]
        nx, nu = self.nx, self.nu
        dyn = zn[:nx] - z[:nx] - z[nx : nx + nu].sum()
        parts_g = ([z[:nx]] if self.first else []) + [dyn, z[nx:]]
        parts_l = ([p] if self.first else []) + [np.zeros(nx), np.full(nu, -self.u_max)]
        parts_u = ([p] if self.first else []) + [np.zeros(nx), np.full(nu, self.u_max)]
        return cost, np.concatenate(parts_g), np.concatenate(parts_l), np.concatenate(parts_u)


def make_problem(cls: problems.MPCClass) -> SparseMPCProblem:
    n = cls.horizon
    stages = tuple(LinearStage(k, cls.nx, cls.nu, terminal=(k == n), first=(k == 0), next_terminal=(k == n - 1),
                               u_max=cls.u_max) for k in range(n + 1))
    return SparseMPCProblem(stages)


@dataclass
class StageData:
    """Per-instance model data: A [B, nx, nx], Bm [B, nx, nu], Q [B, nx], R [B, nu]."""

    a: np.ndarray
    b: np.ndarray
    q: np.ndarray
    r: np.ndarray


def make_data(cls: problems.MPCClass, batch: int, seed: int = 0) -> StageData:
    rng = np.random.default_rng(seed)
    a, b = problems._draw_dynamics(cls, rng, batch)
    q = rng.uniform(1.0, 10.0, (batch, cls.nx))
    r = rng.uniform(0.1, 1.0, (batch, cls.nu))
    f = lambda v: np.ascontiguousarray(v, dtype=np.float32)  # noqa: E731
    return StageData(f(a), f(b), f(q), f(r))


def evaluate_stages(problem: SparseMPCProblem, data, z, params, values_only: bool = False):
    """Every stage's (cost, g, lower, upper, grad, hess, jac) at z (batch-major
    torch tensors, float32), entries in the stage's pattern order; values_only:
    (cost, g, lower, upper)."""
    import torch

    out = []
    dev = z.device
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    A, Bm, Q, R = t(data.a), t(data.b), t(data.q), t(data.r)
    off = 0
    for st in problem.stages:
        nx, nu = st.nx, st.nu
        zk = z[:, off : off + st.z_dim]
        w = Q if st.terminal else torch.cat([Q, R], dim=1)
        grad = w * zk
        cost = 0.5 * (zk * grad).sum(dim=1)
        hess = w.clone()
        if st.terminal:
            e = z.new_zeros((z.shape[0], 0))
            out.append((cost, e, e, e) if values_only else (cost, e, e, e, grad, hess, e))
            break
        zn = z[:, off + st.z_dim : off + st.z_dim + st.next_z_dim]
        x, u = zk[:, :nx], zk[:, nx:]
        dyn = zn[:, :nx] - torch.einsum("bij,bj->bi", A, x) - torch.einsum("bij,bj->bi", Bm, u)
        g = [x] if st.first else []
        g += [dyn, u]
        lo = ([params[:, :nx]] if st.first else []) + [z.new_zeros((z.shape[0], nx)),
                                                       z.new_full((z.shape[0], nu), -st.u_max)]
        up = ([params[:, :nx]] if st.first else []) + [z.new_zeros((z.shape[0], nx)),
                                                       z.new_full((z.shape[0], nu), st.u_max)]
        vals = (cost, torch.cat(g, 1), torch.cat(lo, 1), torch.cat(up, 1))
        if values_only:
            out.append(vals)
        else:
            jac = [z.new_ones((z.shape[0], nx))] if st.first else []
            dyn_j = torch.cat([-A, -Bm, z.new_ones((z.shape[0], nx, 1))], dim=2).reshape(z.shape[0], -1)
            jac += [dyn_j, z.new_ones((z.shape[0], nu))]
            out.append(vals + (grad, hess, torch.cat(jac, 1)))
        off += st.z_dim
    return out


def make_evaluator(problem: SparseMPCProblem, data: StageData, device):
    """The model callable of SparseMPCSQP: evaluate(z, params, values_only).
    The model data are moved to the device once."""
    import torch

    dev_data = StageData(*(torch.as_tensor(v, device=device) for v in (data.a, data.b, data.q, data.r)))

    def evaluate(z, params, values_only):
        return evaluate_stages(problem, dev_data, z, params, values_only)

    return evaluate
