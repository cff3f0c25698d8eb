"""The reference's adjoint derivative path on the CUDA kernels (parity mode).

Mirror of ``adjoint_derivative_compute`` / ``_get_vec`` / ``_get_mat`` of
``compile_osqp(..., derivatives=True)`` (``warpmpc/jax_osqp/solver.py``
1046-1192): the quasi-definite augmented adjoint KKT of the derivative plan
(``build_osqp_plan(..., derivatives=True)``) is assembled per instance,
factored with ``wmpc_factor``, solved with ``wmpc_solve`` and refined
``refinement_iters`` times against the unperturbed matrix (residual by
``wmpc_sym_matvec``), then mapped to the reference's outputs.  The product's
own adjoint (``OSQPEngine.adjoint``, on the forward's factor) does not need
this path; it exists so gradients can be compared with the reference's
algorithm on the same device, arrays and precision.

Assembly and the final index maps are tensor gathers and scatters; the
factorization, the solves and the refinement residuals are the library's
kernels.  Symbolic-major working layout (values ``(nnz, B)``, vectors
``(dim, B)``), batch-major inputs and outputs as the reference's API.
"""

from __future__ import annotations

import numpy as np

from .. import native
from ..jax_qdldl.core import _as_f32, compile_qdldl_cuda
from .types import FixedOSQPPlan

REFINEMENT_ITERS = 100  # the reference's derivative_refinement_iters default


def _row_table(upper):
    """Full-symmetric row table of an upper-CSC pattern: per row, (value
    position, column) of every term of (S x)_row, in CSC order of the terms."""
    cols = np.repeat(np.arange(upper.shape[1]), np.diff(upper.indptr))
    rows = upper.indices.astype(np.int64)
    pos = np.arange(rows.size)
    off = rows != cols
    t_row = np.concatenate([rows, cols[off]])
    t_col = np.concatenate([cols, rows[off]])
    t_pos = np.concatenate([pos, pos[off]])
    o = np.lexsort((t_col, t_row))
    row_ptr = np.zeros(upper.shape[0] + 1, dtype=np.int64)
    np.add.at(row_ptr, t_row + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), t_pos[o].astype(np.int32), t_col[o].astype(np.int32)


class ReferenceAdjoint:
    """Reference-algorithm adjoint of one plan on one device."""

    def __init__(self, plan: FixedOSQPPlan, device=None, refinement_iters: int = REFINEMENT_ITERS):
        import torch

        dp = plan.derivative_plan
        if dp is None:
            raise ValueError("call build_osqp_plan(..., derivatives=True) before using the reference adjoint")
        self.plan, self.dp, self.iters = plan, dp, int(refinement_iters)
        self.qdldl = compile_qdldl_cuda(dp.qdldl_plan, device=device)
        dev = self.qdldl.device_plan.torch_device
        self.device = dev
        it = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64), device=dev)  # noqa: E731
        self.lower, self.upper, self.eq = it(dp.lower_indices), it(dp.upper_indices), it(dp.eq_indices)
        self.g_rows, self.g_cols, self.g_map = it(dp.g_rows), it(dp.g_cols), it(dp.g_a_value_map)
        self.g_sign = torch.as_tensor(np.asarray(dp.g_sign, dtype=np.float32), device=dev)
        self.aeq_map, self.pf_map = it(dp.aeq_a_value_map), it(dp.p_full_value_map)
        self.pos = {k: it(getattr(dp, k)) for k in ("diag_first_pos", "diag_second_pos", "p_block_pos", "g_block_pos",
                                                   "aeq_block_pos", "glambda_block_pos", "slack_diag_pos",
                                                   "aeq_t_block_pos")}
        self.base = torch.as_tensor(np.asarray(dp.adjoint_upper.data, dtype=np.float32), device=dev)
        rp, ep, ec = _row_table(dp.adjoint_upper)
        i32 = lambda a: torch.as_tensor(a, dtype=torch.int32, device=dev)  # noqa: E731
        self.row_ptr, self.ent_pos, self.ent_col = i32(rp), i32(ep), i32(ec)
        self.p_up_rows, self.p_up_cols = it(dp.p_upper_rows), it(dp.p_upper_cols)
        self.a_rows, self.a_cols = it(plan.a_rows), it(plan.a_cols)

    def _matvec_residual(self, values, x, r):
        """K0 x - r, symbolic-major."""
        import torch

        out = torch.empty_like(x)
        native.check(native.lib().wmpc_sym_matvec(
            self.row_ptr.data_ptr(), self.ent_pos.data_ptr(), self.ent_col.data_ptr(), int(x.shape[0]),
            values.data_ptr(), int(values.shape[1]), x.data_ptr(), r.data_ptr(), out.data_ptr(), int(x.shape[1]),
            native.current_stream_handle(self.device)))
        return out

    def compute(self, p_values, a_values, l, u, x, y, dx, dy):
        """adjoint_derivative_compute (solver.py:1047-1156): returns the state
        ``(sol, y_l, y_u, ryl, ryu)``, batch-major."""
        import torch

        pl, dp, dev = self.plan, self.dp, self.device
        f = lambda t, w, name: _as_f32(t, dev, name).reshape(-1, w)  # noqa: E731
        p, a = f(p_values, pl.nnz_p, "p_values"), f(a_values, pl.nnz_a, "a_values")
        l, u, x, y = f(l, pl.m, "l"), f(u, pl.m, "u"), f(x, pl.n, "x"), f(y, pl.m, "y")
        dx, dy = f(dx, pl.n, "dx"), f(dy, pl.m, "dy")
        batch = max(t.shape[0] for t in (p, a, l, u, x, y, dx, dy))
        p, a, l, u, x, y, dx, dy = (t.expand(batch, t.shape[1]) for t in (p, a, l, u, x, y, dx, dy))
        n, nl, ni, ne, half, dim = pl.n, dp.n_ineq_l, dp.n_ineq, dp.n_eq, dp.half_dim, dp.adjoint_dim

        y_u = torch.clamp(y, min=0.0)
        y_l = -torch.clamp(y, max=0.0)
        lam = torch.cat([y_l[:, self.lower], y_u[:, self.upper]], dim=1)
        g_vals = a[:, self.g_map] * self.g_sign[None, :]
        aeq_vals = a[:, self.aeq_map]
        g_x = torch.zeros((batch, ni), dtype=torch.float32, device=dev)
        g_x.index_add_(1, self.g_rows, g_vals * x[:, self.g_cols])
        slacks = g_x - torch.cat([-l[:, self.lower], u[:, self.upper]], dim=1)

        k0 = self.base[None, :].expand(batch, -1).clone()
        k0[:, self.pos["diag_first_pos"]] = 1.0
        k0[:, self.pos["diag_second_pos"]] = 0.0
        k0[:, self.pos["p_block_pos"]] = p[:, self.pf_map]
        k0[:, self.pos["g_block_pos"]] = g_vals
        k0[:, self.pos["aeq_block_pos"]] = aeq_vals
        k0[:, self.pos["glambda_block_pos"]] = lam[:, self.g_rows] * g_vals
        k0[:, self.pos["slack_diag_pos"]] = slacks
        k0[:, self.pos["aeq_t_block_pos"]] = aeq_vals
        k = k0.clone()
        k[:, self.pos["diag_first_pos"]] = float(np.float32(1.0) + np.float32(dp.eps))  # 1 + eps in float32
        k[:, self.pos["diag_second_pos"]] = -float(np.float32(dp.eps))

        rhs = torch.zeros((batch, dim), dtype=torch.float32, device=dev)
        rhs[:, :n] = -dx
        rhs[:, n : n + nl] = -dy[:, self.lower]
        rhs[:, n + nl : n + ni] = -dy[:, self.upper]
        d_nu = torch.where(y[:, self.eq] >= 0.0, dy[:, self.eq], -dy[:, self.eq])
        rhs[:, n + ni : n + ni + ne] = -d_nu

        k0_s, k_s, rhs_s = k0.t().contiguous(), k.t().contiguous(), rhs.t().contiguous()
        lx, _, dinv = self.qdldl.factor(k_s)
        sol = self.qdldl.solve(lx, dinv, rhs_s)
        for _ in range(self.iters):
            sol = sol - self.qdldl.solve(lx, dinv, self._matvec_residual(k0_s, sol, rhs_s))
        sol = sol.t().contiguous()

        m = pl.m
        r_yl = torch.zeros((batch, m), dtype=torch.float32, device=dev)
        r_yu = torch.zeros((batch, m), dtype=torch.float32, device=dev)
        pos = half + n
        r_yl[:, self.lower] = -sol[:, pos : pos + nl]
        pos += nl
        r_yu[:, self.upper] = sol[:, pos : pos + dp.n_ineq_u]
        pos += dp.n_ineq_u
        eq_sol = sol[:, pos : pos + ne]
        eq_y = y[:, self.eq]
        positive = eq_y >= 0.0
        r_yu[:, self.eq] = torch.where(positive, eq_sol / eq_y, torch.zeros_like(eq_sol))
        r_yl[:, self.eq] = torch.where(positive, torch.zeros_like(eq_sol), -eq_sol / eq_y)
        return sol, y_l, y_u, -(r_yl * y_l), r_yu * y_u

    def get_vec(self, state):
        """adjoint_derivative_get_vec (solver.py:1158-1164): (dq, dl, du)."""
        sol, _, _, ryl, ryu = state
        half, n = self.dp.half_dim, self.plan.n
        return sol[:, half : half + n], ryl, -ryu

    def get_mat(self, x, y, state):
        """adjoint_derivative_get_mat (solver.py:1166-1192): (dP on P's upper pattern, dA on A's)."""
        sol, y_l, y_u, ryl, ryu = state
        half, n = self.dp.half_dim, self.plan.n
        rx = sol[:, half : half + n]
        x = _as_f32(x, self.device, "x").reshape(-1, n).expand(rx.shape[0], n)
        d_p = 0.5 * (rx[:, self.p_up_rows] * x[:, self.p_up_cols] + rx[:, self.p_up_cols] * x[:, self.p_up_rows])
        d_a = ((y_u[:, self.a_rows] - y_l[:, self.a_rows]) * rx[:, self.a_cols]
               + (ryu[:, self.a_rows] - ryl[:, self.a_rows]) * x[:, self.a_cols])
        return d_p, d_a
