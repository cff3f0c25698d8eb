"""Nonlinear SQP workload: rigid-body quadrotor MPC with RK4 dynamics.

Twelve states ``[p (3), roll/pitch/yaw (3), v (3), w (3)]``, four motor
thrusts ``0 <= u <= 0.15 N``, mass 0.03 kg, inertia diag(1.4e-5, 1.4e-5,
2.2e-5) kg m^2, one classical RK4 step of dt = 0.02 s per stage (the model
and its equations: ``wmpc_quadrotor_rk4`` in include/warpmpc_b200.h), horizon
N stages.  Stage k < N has variables ``z_k = [x_k, u_k]``; the terminal
stage ``z_N = x_N``.  Cost ``0.5 (x - x_ref)' Q (x - x_ref) + 0.5 (u -
u_hover)' R (u - u_hover)`` (terminal: ``Q``; x_ref the hover point at the
origin, u_hover = m g / 4), with per-instance diagonal weights.
Constraints: stage 0 pins ``x_0 = x0`` (the instance's parameters); every
stage k < N has the dynamics ``x_{k+1} - F(x_k, u_k) = 0`` and the thrust box.

The stage layout is the reference's stage-function interface (grad, Hessian
and Jacobian values in each stage's pattern order, as its CasADi stages
deliver them: ``warpmpc/jax_sqp/casadi_stage.py:66-189``; like them the QP's
P is the cost Hessian, ``casadi_stage.py:119``).  The dynamics and their
Jacobian come from the CUDA model kernel (forward-mode derivatives); the
rest of a stage's values are formed with torch on the device.

``QuadrotorSQP`` runs the workload: SQP iterations with the filter line
search (``SparseMPCSQP``), warm-started QP solves, capturable in one CUDA
graph, and the gradient of a loss on the final iterate's first input with
respect to x0 and the cost weights through the last QP (the adjoint on the
kept factorization, no refactorization), holding the last linearization
point and step length fixed.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import native
from .jax_osqp import OSQPSettings
from .jax_sqp import SparseMPCSQP, build_sparse_mpc_plan
from .jax_sqp.assembly import SparseMPCProblem

NX, NU = 12, 4
MASS, GRAVITY = 0.03, 9.81
INERTIA = (1.4e-5, 1.4e-5, 2.2e-5)
ARM = 0.046 / np.sqrt(2.0)
YAW_COEF = 0.006
DT = 0.02
U_MAX = 0.15
U_HOVER = MASS * GRAVITY / 4.0
# nominal diagonal weights (each instance scales them by U[0.5, 1.5])
Q_NOMINAL = np.array([10.0, 10.0, 10.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.1, 0.1, 0.1])
R_NOMINAL = np.full(NU, 500.0)


def model_struct():
    return native.QuadrotorModel(mass=MASS, jx=INERTIA[0], jy=INERTIA[1], jz=INERTIA[2], arm=ARM, yaw_coef=YAW_COEF,
                                 gravity=GRAVITY)


def jac_pattern():
    """(cols [126], row_ptr [13]) of the dynamics rows' entries, as the kernel writes them."""
    cols = np.empty(126, dtype=np.int32)
    ptr = np.empty(NX + 1, dtype=np.int32)
    native.check(native.lib().wmpc_quadrotor_jac_pattern(native.ptr_i32(cols), native.ptr_i32(ptr)))
    return cols, ptr


@dataclass(frozen=True)
class RK4Stage:
    """One stage's fixed local sparsity (the attributes the SQP planner reads)."""

    k: int
    terminal: bool
    first: bool
    next_terminal: bool

    nx = NX
    nu = NU

    @property
    def has_next(self):
        return not self.terminal

    @property
    def z_dim(self):
        return NX if self.terminal else NX + NU

    @property
    def next_z_dim(self):
        if self.terminal:
            return 0
        return NX if self.next_terminal else NX + NU

    @property
    def param_dim(self):
        return NX if self.first else 0

    @property
    def constraint_dim(self):
        return 0 if self.terminal else (NX if self.first else 0) + NX + NU

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
        """[x0 rows (stage 0): identity], dynamics rows (the kernel's order), input rows."""
        rows, cols = [], []
        r0 = 0
        if self.first:
            rows += list(range(NX))
            cols += list(range(NX))
            r0 = NX
        jc, jp = jac_pattern()
        for r in range(NX):
            for e in range(jp[r], jp[r + 1]):
                rows.append(r0 + r)
                cols.append(int(jc[e]))  # 16 + r is x_{k+1, r}: local column z_dim + r
        for j in range(NU):
            rows.append(r0 + NX + j)
            cols.append(NX + j)
        return np.asarray(rows, dtype=np.int32), np.asarray(cols, dtype=np.int32)

    @property
    def jac_rows(self):
        return self._jac_pattern()[0] if not self.terminal else np.zeros(0, np.int32)

    @property
    def jac_cols(self):
        return self._jac_pattern()[1] if not self.terminal else np.zeros(0, np.int32)

    def value_function(self, z, *rest):
        """(cost, g, lower, upper) with the bounds this stage always has (the
        planner reads only the bound types; the values come from the kernel)."""
        p = rest[-1]
        if self.terminal:
            return 0.0, np.zeros(0), np.zeros(0), np.zeros(0)
        parts_g = ([z[:NX]] if self.first else []) + [np.zeros(NX), z[NX:]]
        parts_l = ([p] if self.first else []) + [np.zeros(NX), np.zeros(NU)]
        parts_u = ([p] if self.first else []) + [np.zeros(NX), np.full(NU, U_MAX)]
        return 0.0, np.concatenate(parts_g), np.concatenate(parts_l), np.concatenate(parts_u)


def make_problem(horizon: int) -> SparseMPCProblem:
    return SparseMPCProblem(tuple(RK4Stage(k, terminal=(k == horizon), first=(k == 0),
                                           next_terminal=(k == horizon - 1)) for k in range(horizon + 1)))


@dataclass
class QuadrotorData:
    """Per-instance parameters: x0 [B, 12], weights Q [B, 12], R [B, 4]."""

    x0: np.ndarray
    q: np.ndarray
    r: np.ndarray


def make_data(batch: int, seed: int = 0) -> QuadrotorData:
    """x0: position U[-1, 1] m, attitude U[-0.3, 0.3] rad, velocities and
    body rates U[-0.5, 0.5]; weights: the nominal ones scaled by U[0.5, 1.5]."""
    rng = np.random.default_rng(seed)
    x0 = np.concatenate([rng.uniform(-1, 1, (batch, 3)), rng.uniform(-0.3, 0.3, (batch, 3)),
                         rng.uniform(-0.5, 0.5, (batch, 3)), rng.uniform(-0.5, 0.5, (batch, 3))], axis=1)
    q = Q_NOMINAL[None] * rng.uniform(0.5, 1.5, (batch, NX))
    r = R_NOMINAL[None] * rng.uniform(0.5, 1.5, (batch, NU))
    f = lambda v: np.ascontiguousarray(v, dtype=np.float32)  # noqa: E731
    return QuadrotorData(f(x0), f(q), f(r))


def initial_guess(plan, x0):
    """z with every state at x0 and every input at hover (torch, on x0's device)."""
    import torch

    batch = x0.shape[0]
    n_stages = len(plan.stage_var_dims) - 1
    blocks = [torch.cat([x0, x0.new_full((batch, NU), U_HOVER)], 1)] * n_stages + [x0]
    return torch.cat(blocks, 1).contiguous()


class Evaluator:
    """The model callable of SparseMPCSQP: ``evaluate(z, params, values_only)``
    with params = x0 (batch-major torch tensors on the device)."""

    def __init__(self, problem: SparseMPCProblem, q, r, device):
        import torch

        self.problem = problem
        self.device = torch.device(device)
        self.q = torch.as_tensor(q, device=self.device, dtype=torch.float32)
        self.r = torch.as_tensor(r, device=self.device, dtype=torch.float32)
        self.n_stages = len(problem.stages) - 1
        self.model = model_struct()
        self.lib = native.lib()

    def dynamics(self, z, with_jac):
        """(x_next [N, B, 12], jac [N, B, 126] or None) from the CUDA model kernel."""
        import torch

        batch = z.shape[0]
        z = z.contiguous()
        xn = torch.empty((self.n_stages, batch, NX), dtype=torch.float32, device=self.device)
        jac = torch.empty((self.n_stages, batch, 126), dtype=torch.float32, device=self.device) if with_jac else None
        native.check(self.lib.wmpc_quadrotor_rk4(ctypes.byref(self.model), z.data_ptr(), z.stride(0), batch,
                                                 self.n_stages, np.float32(DT), xn.data_ptr(),
                                                 jac.data_ptr() if jac is not None else None,
                                                 native.current_stream_handle(self.device)))
        return xn, jac

    def __call__(self, z, params, values_only):
        import torch

        xn, jac = self.dynamics(z, not values_only)
        batch = z.shape[0]
        out = []
        zeros = z.new_zeros((batch, NX))
        u_lo, u_hi = z.new_zeros((batch, NU)), z.new_full((batch, NU), U_MAX)
        for st in self.problem.stages:
            off = NX_NU * st.k
            x = z[:, off : off + NX]
            if st.terminal:
                grad = self.q * x
                cost = 0.5 * (x * grad).sum(1)
                e = z.new_zeros((batch, 0))
                out.append((cost, e, e, e) if values_only else (cost, e, e, e, grad, self.q, e))
                break
            u = z[:, off + NX : off + NX_NU]
            du = u - U_HOVER
            gx, gu = self.q * x, self.r * du
            cost = 0.5 * ((x * gx).sum(1) + (du * gu).sum(1))
            x_next = z[:, off + NX_NU : off + NX_NU + NX]
            g = ([x] if st.first else []) + [x_next - xn[st.k], u]
            lo = ([params] if st.first else []) + [zeros, u_lo]
            up = ([params] if st.first else []) + [zeros, u_hi]
            vals = (cost, torch.cat(g, 1), torch.cat(lo, 1), torch.cat(up, 1))
            if values_only:
                out.append(vals)
            else:
                j = ([z.new_ones((batch, NX))] if st.first else []) + [jac[st.k], z.new_ones((batch, NU))]
                out.append(vals + (torch.cat([gx, gu], 1), torch.cat([self.q, self.r], 1), torch.cat(j, 1)))
        return out


NX_NU = NX + NU


def default_settings(max_iter: int = 25) -> OSQPSettings:
    return OSQPSettings(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=max_iter, scaling=10, rho_is_vec=True,
                        check_termination=0)


class _RepresentativeStage:
    """A stage with the values at the hover point (from the model kernel) as
    ``sparse_function`` output: the representative P/A/q the QP's scaling is
    computed from."""

    def __init__(self, stage, raw):
        self._stage, self._raw = stage, raw

    def __getattr__(self, name):
        return getattr(self._stage, name)

    def sparse_function(self, *args):
        return self._raw


def build_plan(horizon: int, device, settings: OSQPSettings | None = None, derivatives: bool = False):
    """The SQP plan of the workload, scaled from the hover trajectory (the
    stage values there come from the model kernel on `device`)."""
    import torch

    problem = make_problem(horizon)
    q = torch.as_tensor(Q_NOMINAL[None], dtype=torch.float32, device=device)
    r = torch.as_tensor(R_NOMINAL[None], dtype=torch.float32, device=device)
    ev = Evaluator(problem, q, r, device)
    n_z = NX_NU * horizon + NX
    z_ref = torch.zeros((1, n_z), device=device)
    for k in range(horizon):
        z_ref[:, NX_NU * k + NX : NX_NU * (k + 1)] = U_HOVER
    vals = ev(z_ref, torch.zeros((1, NX), device=device), False)
    stages = []
    for st, v in zip(problem.stages, vals):
        raw = tuple(np.asarray(t.detach().cpu().numpy()[0], dtype=np.float64) for t in v)
        stages.append(_RepresentativeStage(st, raw))
    rep = SparseMPCProblem(tuple(stages))
    plan = build_sparse_mpc_plan(rep, osqp_settings=settings or default_settings(), derivatives=derivatives,
                                 representative_z=z_ref.cpu().numpy()[0], representative_params=np.zeros(NX))
    return problem, plan


class QuadrotorSQP:
    """The nonlinear SQP workload on one device: ``iterations`` SQP steps with
    the filter line search from the hover initial guess, each QP warm-started
    from the previous one, and the gradient of ``||u0 - u_target||^2`` (u0 the
    first input of the final iterate) with respect to x0 and the weights."""

    def __init__(self, horizon: int, data: QuadrotorData, device, iterations: int = 5, max_iter: int = 25):
        import torch

        self.device = torch.device(device)
        self.horizon, self.iterations = horizon, iterations
        self.problem, self.plan = build_plan(horizon, self.device, default_settings(max_iter))
        t = lambda a: torch.as_tensor(a, device=self.device, dtype=torch.float32)  # noqa: E731
        self.x0, q, r = t(data.x0), t(data.q), t(data.r)
        self.evaluator = Evaluator(self.problem, q, r, self.device)
        self.sqp = SparseMPCSQP(self.problem, self.plan, self.evaluator, device=self.device)
        self.q_cols = [np.asarray(a.q_cols, dtype=np.int64) for a in self.plan.assemblies]
        self.p_pos = [np.asarray(a.p_pos, dtype=np.int64) for a in self.plan.assemblies]
        # the same indices on the device, states and inputs apart (gradient's gathers, graph-capturable)
        ix = lambda a: torch.as_tensor(a, dtype=torch.int64, device=self.device)  # noqa: E731
        self._grad_index = [(ix(c[:NX]), ix(p[:NX]), ix(c[NX:]), ix(p[NX:])) for c, p in zip(self.q_cols, self.p_pos)]

    def solve(self, keep_factor: bool = False):
        """The SQP iterations; returns (z, last step result).  With
        keep_factor the last QP keeps its factorization for ``gradient``."""
        z = initial_guess(self.plan, self.x0)
        warm = None
        r = None
        for it in range(self.iterations):
            last = it == self.iterations - 1
            r = self.sqp.line_search_step(z, self.x0, warm, keep_factor=keep_factor and last)
            z = r.z_next
            warm = (r.solve.direction, r.solve.z, r.solve.y)
        return z, r

    def gradient(self, z, r, u_target):
        """d ||u0 - u_target||^2 / d (x0 [B, 12], Q [B, 12], R [B, 4]) through the last QP."""
        import torch

        eng = self.sqp.qp.engine
        lin = r.solve.linearization
        step = r.line_search.step_length.reshape(-1, 1)
        dz = torch.zeros_like(z)
        dz[:, NX : NX_NU] = 2.0 * (z[:, NX : NX_NU] - u_target)
        dx = (step * dz).contiguous()  # z_next = z_lin + step d
        dq, dl, du, dp, _ = eng.adjoint(eng.last_workspace, lin.p_values, lin.a_values, lin.l, lin.u,
                                        r.solve.direction, r.solve.z, r.solve.y, dx, None)
        z_lin = z - step * r.solve.direction
        g_x0 = dl[:, :NX] + du[:, :NX]  # l = u = x0 - x_lin0 on the first rows
        g_q = torch.zeros_like(self.evaluator.q)
        g_r = torch.zeros_like(self.evaluator.r)
        for k, st in enumerate(self.problem.stages):
            off = NX_NU * k
            cx, px, cu, pu = self._grad_index[k]
            # P's diagonal entry of a variable is its weight; q's entry the weight times its offset
            g_q += dp[:, px] + dq[:, cx] * z_lin[:, off : off + NX]
            if not st.terminal:
                g_r += dp[:, pu] + dq[:, cu] * (z_lin[:, off + NX : off + NX_NU] - U_HOVER)
        return g_x0, g_q, g_r
