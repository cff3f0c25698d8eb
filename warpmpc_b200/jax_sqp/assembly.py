"""Sparse MPC QP assembly: the plan and the batched linearization on the GPU.

Mirror of ``build_sparse_mpc_plan`` (``warpmpc/jax_sqp/sparse_mpc.py:532-691``,
with ``_offsets`` 181-184, ``_csc_pattern`` 196-211, ``_stage_bound_samples``
476-491, ``_classify_problem_bounds`` 494-518, ``_local_to_global`` 521-529)
and of the assembly half of ``_linearize_jit`` (``sparse_mpc.py:855-901``):
every stage's evaluated cost, constraint values and bounds, gradient, Hessian
and Jacobian values are scattered into the QP ``(P, A, q, l = lower - g,
u = upper - g)`` and the record ``SQPLinearization``.

The reference evaluates its stages with CasADi-generated functions; the
stage *evaluation* stays the caller's here (any object with the attributes
below, a reference ``CasadiStageFunction`` included), and the assembly runs
in one kernel (``wmpc_sqp_assemble``): per output entry the list of stage
values that add into it, summed in stage order -- the order of the
reference's per-stage scatter-adds -- so the result is deterministic and
equals a float32 sequential restatement bit for bit.

A stage description needs: ``has_next``, ``z_dim``, ``next_z_dim``,
``param_dim``, ``constraint_dim``, ``grad_cols``, ``hess_rows``,
``hess_cols``, ``jac_rows``, ``jac_cols`` and ``value_function(z, [zn,] p)
-> (cost, g, lower, upper)`` (bound classification);
``sparse_function`` (``raw[4:7]`` = grad, hess, jac values) only when
representative values are given.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple, Sequence

import numpy as np
import scipy.sparse as sp

from .. import native
from ..jax_osqp import OSQPSettings, build_osqp_plan

OSQP_INFTY = 1e30
OSQP_MIN_SCALING = 1e-4


@dataclass(frozen=True)
class SparseMPCProblem:
    """A stage-ordered MPC problem with fixed local sparsity (sparse_mpc.py:70-75)."""

    stages: tuple


@dataclass(frozen=True)
class StageAssembly:
    """Global scatter maps of one stage's derivative values (types.py:56-66)."""

    z_offset: int
    next_z_offset: int
    param_offset: int
    constraint_offset: int
    q_cols: np.ndarray
    p_pos: np.ndarray
    a_pos: np.ndarray


@dataclass(frozen=True)
class SparseMPCPlan:
    """Fixed sparsity and index data of an MPC SQP problem (types.py:69-84)."""

    stage_var_dims: tuple
    param_dims: tuple
    constraint_dims: tuple
    z_offsets: np.ndarray
    param_offsets: np.ndarray
    constraint_offsets: np.ndarray
    p_pattern: sp.csc_matrix
    a_pattern: sp.csc_matrix
    representative_l: np.ndarray
    representative_u: np.ndarray
    osqp_plan: object
    assemblies: tuple


class SQPLinearization(NamedTuple):
    """Batched QP data of one SQP linearization (types.py:14-25)."""

    p_values: object
    a_values: object
    q: object
    l: object
    u: object
    cost: object
    g: object
    constraint_l: object
    constraint_u: object


def _offsets(widths: Sequence[int]) -> np.ndarray:
    out = np.zeros(len(widths) + 1, dtype=np.int32)
    out[1:] = np.cumsum(np.asarray(widths, dtype=np.int32))
    return out


def _pattern(shape, rows, cols):
    """Sorted unique (row, col) keys as a CSC pattern; position of every key."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    key = cols * shape[0] + rows
    uniq = np.unique(key)  # CSC order: by column, then row
    matrix = sp.csc_matrix((np.zeros(uniq.size), ((uniq % shape[0]).astype(np.int32), (uniq // shape[0]).astype(np.int32))),
                           shape=shape)
    matrix.sort_indices()
    return matrix, uniq


def _positions(uniq, shape, rows, cols):
    key = np.asarray(cols, dtype=np.int64) * shape[0] + np.asarray(rows, dtype=np.int64)
    return np.searchsorted(uniq, key).astype(np.int32)


def _bound_samples(stage):
    """Stage bounds at the probes z = p = 0, 1, -1 (sparse_mpc.py:476-491)."""
    lowers, uppers = [], []
    for fill in (0.0, 1.0, -1.0):
        z = np.full(stage.z_dim, fill)
        p = np.full(stage.param_dim, fill)
        if stage.has_next:
            _, _, lo, up = stage.value_function(z, np.full(stage.next_z_dim, fill), p)
        else:
            _, _, lo, up = stage.value_function(z, p)
        lowers.append(np.asarray(lo, dtype=np.float64).reshape(-1))
        uppers.append(np.asarray(up, dtype=np.float64).reshape(-1))
    return np.stack(lowers), np.stack(uppers)


def classify_problem_bounds(problem: SparseMPCProblem):
    """Representative bounds with each row's fixed type (sparse_mpc.py:494-518):
    equality rows 0/0, lower-bounded 0, upper-bounded 1, else +-1e30."""
    lo_parts, up_parts = [], []
    thr = OSQP_INFTY * OSQP_MIN_SCALING
    for stage in problem.stages:
        ls, us = _bound_samples(stage)
        equal = np.all(np.isclose(ls, us, rtol=1e-9, atol=1e-9), axis=0)
        lower = np.where(np.any(ls > -thr, axis=0), 0.0, -OSQP_INFTY)
        upper = np.where(np.any(us < thr, axis=0), 1.0, OSQP_INFTY)
        lower[equal] = 0.0
        upper[equal] = 0.0
        lo_parts.append(lower)
        up_parts.append(upper)
    return np.concatenate(lo_parts), np.concatenate(up_parts)


def _local_to_global(stage, z_offset, next_z_offset):
    own = z_offset + np.arange(stage.z_dim, dtype=np.int32)
    if not stage.has_next:
        return own
    return np.concatenate([own, next_z_offset + np.arange(stage.next_z_dim, dtype=np.int32)])


def build_sparse_mpc_plan(problem: SparseMPCProblem, *, osqp_settings: OSQPSettings | None = None,
                          derivatives: bool = False, representative_z=None, representative_params=None):
    """Fixed index data for the batched QP assembly (sparse_mpc.py:532-691)."""
    stages = problem.stages
    if len(stages) < 2:
        raise ValueError("MPC SQP needs at least one transition and one terminal stage")
    for i, st in enumerate(stages[:-1]):
        if not st.has_next:
            raise ValueError(f"stage {i} must have a next-stage input")
    if stages[-1].has_next:
        raise ValueError("terminal stage must not have a next-stage input")
    var_dims = [stages[0].z_dim] + [st.next_z_dim for st in stages[:-1]]
    for i, (want, st) in enumerate(zip(var_dims, stages)):
        if st.z_dim != want:
            raise ValueError(f"stage {i} z_dim={st.z_dim} does not match expected {want}")
    z_off = _offsets(var_dims)
    p_off = _offsets([st.param_dim for st in stages])
    c_off = _offsets([st.constraint_dim for st in stages])
    nz, nc = int(z_off[-1]), int(c_off[-1])

    q_cols, p_keys, a_keys = [], [], []
    for i, st in enumerate(stages):
        lg = _local_to_global(st, int(z_off[i]), int(z_off[i + 1]) if st.has_next else 0)
        q_cols.append(lg[np.asarray(st.grad_cols, dtype=np.int64)])
        hr = lg[np.asarray(st.hess_rows, dtype=np.int64)]
        hc = lg[np.asarray(st.hess_cols, dtype=np.int64)]
        p_keys.append((np.minimum(hr, hc), np.maximum(hr, hc)))  # upper triangle
        a_keys.append((int(c_off[i]) + np.asarray(st.jac_rows, dtype=np.int64),
                       lg[np.asarray(st.jac_cols, dtype=np.int64)]))
    diag = np.arange(nz)
    p_pattern, p_uniq = _pattern((nz, nz), np.concatenate([diag] + [k[0] for k in p_keys]),
                                 np.concatenate([diag] + [k[1] for k in p_keys]))
    a_rows_all = np.concatenate([k[0] for k in a_keys]) if a_keys else np.zeros(0, np.int64)
    a_cols_all = np.concatenate([k[1] for k in a_keys]) if a_keys else np.zeros(0, np.int64)
    a_pattern, a_uniq = _pattern((nc, nz), a_rows_all, a_cols_all)
    assemblies = tuple(
        StageAssembly(
            z_offset=int(z_off[i]), next_z_offset=int(z_off[i + 1]) if st.has_next else 0,
            param_offset=int(p_off[i]), constraint_offset=int(c_off[i]),
            q_cols=np.asarray(q_cols[i], dtype=np.int32),
            p_pos=_positions(p_uniq, (nz, nz), *p_keys[i]),
            a_pos=_positions(a_uniq, (nc, nz), *a_keys[i]),
        )
        for i, st in enumerate(stages)
    )
    settings = osqp_settings or OSQPSettings(rho=0.1, sigma=1e-6, alpha=1.6, max_iter=25, scaling=0,
                                             rho_is_vec=False, check_termination=0)
    lower0, upper0 = classify_problem_bounds(problem)

    p_for, a_for, scaling_q = p_pattern, a_pattern, None
    if (representative_z is None) != (representative_params is None):
        raise ValueError("representative_z and representative_params must be provided together")
    if representative_z is not None:
        z_ref = np.asarray(representative_z, dtype=np.float64)
        p_ref = np.asarray(representative_params, dtype=np.float64)
        z_ref = z_ref[0] if z_ref.ndim == 2 else z_ref
        p_ref = p_ref[0] if p_ref.ndim == 2 else p_ref
        if z_ref.shape != (nz,):
            raise ValueError(f"representative_z must have shape {(nz,)}, got {z_ref.shape}")
        if p_ref.shape != (int(p_off[-1]),):
            raise ValueError(f"representative_params must have shape {(int(p_off[-1]),)}, got {p_ref.shape}")
        pv, av, qv = np.zeros(p_pattern.nnz), np.zeros(a_pattern.nnz), np.zeros(nz)
        for st, asm in zip(stages, assemblies):
            zs = z_ref[asm.z_offset : asm.z_offset + st.z_dim]
            ps = p_ref[asm.param_offset : asm.param_offset + st.param_dim]
            if st.has_next:
                raw = st.sparse_function(zs, z_ref[asm.next_z_offset : asm.next_z_offset + st.next_z_dim], ps)
            else:
                raw = st.sparse_function(zs, ps)
            np.add.at(qv, asm.q_cols, np.asarray(raw[4], dtype=np.float64).reshape(-1))
            np.add.at(pv, asm.p_pos, np.asarray(raw[5], dtype=np.float64).reshape(-1))
            np.add.at(av, asm.a_pos, np.asarray(raw[6], dtype=np.float64).reshape(-1))
        p_for, a_for = p_pattern.copy(), a_pattern.copy()
        p_for.data, a_for.data = pv, av
        scaling_q = qv
    osqp_plan = build_osqp_plan(p_for, a_for, lower0, upper0, settings, derivatives=derivatives,
                                scaling_q=scaling_q)
    return SparseMPCPlan(
        stage_var_dims=tuple(int(v) for v in var_dims), param_dims=tuple(int(st.param_dim) for st in stages),
        constraint_dims=tuple(int(st.constraint_dim) for st in stages), z_offsets=z_off, param_offsets=p_off,
        constraint_offsets=c_off, p_pattern=p_pattern, a_pattern=a_pattern, representative_l=lower0,
        representative_u=upper0, osqp_plan=osqp_plan, assemblies=assemblies,
    )


# ---------------------------------------------------------------------------
# batched assembly on the GPU
# ---------------------------------------------------------------------------

def stage_value_layout(plan: SparseMPCPlan, problem: SparseMPCProblem, values_only: bool = False):
    """Column offsets of each stage's values in the packed per-instance row the
    kernel reads: per stage [cost (1) | g | lower | upper (constraint_dim each)
    | grad | hess | jac] (values_only: without the derivative parts), stages in
    order.  Returns (offsets [stages, 7], width)."""
    offs, col = [], 0
    for st, asm in zip(problem.stages, plan.assemblies):
        nc = st.constraint_dim
        parts = [1, nc, nc, nc] + ([0, 0, 0] if values_only else [asm.q_cols.size, asm.p_pos.size, asm.a_pos.size])
        o = []
        for w in parts:
            o.append(col)
            col += w
        offs.append(o)
    return np.asarray(offs, dtype=np.int64), col


def assembly_tables(plan: SparseMPCPlan, problem: SparseMPCProblem, values_only: bool = False):
    """Gather tables of the assembly kernel.  Output row of one instance:
    [q (n) | P values (nnz_p) | A values (nnz_a)] summed from their sources in
    stage order (``add_ptr``/``add_src``), then the m constraint rows' g,
    lower and upper sources (``row_src``: the g column of each row, then each
    row's stage constraint_dim nc: lower and upper sit nc and 2 nc further),
    and the stages' cost columns.  values_only: no q/P/A outputs (the
    reference's _evaluate_values, sparse_mpc.py:840-853)."""
    offs, width = stage_value_layout(plan, problem, values_only)
    n, nnz_p, nnz_a = int(plan.z_offsets[-1]), plan.p_pattern.nnz, plan.a_pattern.nnz
    if values_only:
        n = nnz_p = nnz_a = 0
    dest, src = [], []
    for s, (st, asm) in enumerate(zip(problem.stages, plan.assemblies)):
        if values_only:
            break
        dest += [asm.q_cols.astype(np.int64), n + asm.p_pos.astype(np.int64), n + nnz_p + asm.a_pos.astype(np.int64)]
        src += [offs[s, 4] + np.arange(asm.q_cols.size), offs[s, 5] + np.arange(asm.p_pos.size),
                offs[s, 6] + np.arange(asm.a_pos.size)]
    dest = np.concatenate(dest) if dest else np.zeros(0, np.int64)
    src = np.concatenate(src) if src else np.zeros(0, np.int64)
    order = np.argsort(dest, kind="stable")  # stage order (then entry order) within each destination
    n_add = n + nnz_p + nnz_a
    add_ptr = np.zeros(n_add + 1, dtype=np.int64)
    np.add.at(add_ptr, dest + 1, 1)
    add_ptr = np.cumsum(add_ptr)
    m = int(plan.constraint_offsets[-1])
    row_src = np.zeros(2 * m, dtype=np.int64)  # [g column of each row | its stage's constraint_dim]
    for s, (st, asm) in enumerate(zip(problem.stages, plan.assemblies)):
        r0 = asm.constraint_offset
        row_src[r0 : r0 + st.constraint_dim] = offs[s, 1] + np.arange(st.constraint_dim)
        row_src[m + r0 : m + r0 + st.constraint_dim] = st.constraint_dim
    cost_src = offs[:, 0].copy()
    return {
        "add_ptr": add_ptr.astype(np.int32), "add_src": src[order].astype(np.int32), "row_src": row_src.astype(np.int32),
        "cost_src": cost_src.astype(np.int32), "width": int(width), "n": n, "nnz_p": nnz_p, "nnz_a": nnz_a,
        "m": int(plan.constraint_offsets[-1]), "stage_offsets": offs,
    }


class QPAssembler:
    """Device tables of one plan; ``assemble(values)`` -> SQPLinearization.
    ``values_only``: stage values without derivatives in, only cost, g and the
    bounds out (q, P and A empty)."""

    def __init__(self, plan: SparseMPCPlan, problem: SparseMPCProblem, device=None, values_only: bool = False):
        import torch

        native.require_cuda()
        self.plan, self.problem, self.values_only = plan, problem, values_only
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        t = assembly_tables(plan, problem, values_only)
        self.tables = t
        i32 = lambda a: torch.as_tensor(a, dtype=torch.int32, device=self.device)  # noqa: E731
        self.add_ptr, self.add_src = i32(t["add_ptr"]), i32(t["add_src"])
        self.row_src, self.cost_src = i32(t["row_src"]), i32(t["cost_src"])
        self.width = t["width"]

    def pack(self, stage_values):
        """Per stage (cost [B], g, lower, upper [B, nc], grad, hess, jac [B, k]) -> the packed [B, width] row."""
        import torch

        cols = []
        for vals in stage_values:
            cost, g, lo, up = vals[:4]
            cols += [cost.reshape(-1, 1), g, lo, up] + ([] if self.values_only else list(vals[4:7]))
        return torch.cat([c.to(self.device, torch.float32) for c in cols], dim=1).contiguous()

    def assemble(self, values) -> SQPLinearization:
        """values: the packed [B, width] float32 rows (``pack``)."""
        import torch

        v = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values, np.float32))
        v = v.to(self.device, torch.float32).contiguous()
        if v.dim() != 2 or v.shape[1] != self.width:
            raise ValueError(f"values must have shape (batch, {self.width})")
        b = int(v.shape[0])
        t = self.tables
        e = lambda *s: torch.empty(*s, dtype=torch.float32, device=self.device)  # noqa: E731
        out = SQPLinearization(e(b, t["nnz_p"]), e(b, t["nnz_a"]), e(b, t["n"]), e(b, t["m"]), e(b, t["m"]), e(b),
                               e(b, t["m"]), e(b, t["m"]), e(b, t["m"]))
        d = native.SqpAssembleDims(b, t["n"], t["nnz_p"], t["nnz_a"], t["m"], len(self.problem.stages), self.width)
        native.check(native.lib().wmpc_sqp_assemble(
            ctypes.byref(d), self.add_ptr.data_ptr(), self.add_src.data_ptr(), self.row_src.data_ptr(),
            self.cost_src.data_ptr(), v.data_ptr(), out.q.data_ptr(), out.p_values.data_ptr(),
            out.a_values.data_ptr(), out.l.data_ptr(), out.u.data_ptr(), out.cost.data_ptr(), out.g.data_ptr(),
            out.constraint_l.data_ptr(), out.constraint_u.data_ptr(), native.current_stream_handle(self.device)))
        return out
