"""Host-side OSQP setup for the fixed-pattern batched solver.

Runs once per pattern: Ruiz equilibration, the per-constraint rho vector, the
KKT pattern ``[[P + sigma I, A^T], [A, -diag(1/rho)]]`` with the maps that
scatter per-instance P/A values into it, and the LDL^T plan of that pattern.
Outputs equal the reference's array-for-array (including float64 scaling
factors, which are computed with the reference's operation order so they
agree to the last bit).

Reference: ``warpmpc/jax_osqp/solver.py`` (``_upper_with_diagonal`` 64-78,
``_build_kkt_and_maps`` 81-150, ``_bounds_type`` 153-161, ``_rho_vectors``
164-183, ``_p_full_pattern`` 186-204, ``_compute_scaling`` 262-343,
``_build_derivative_plan`` 413-571, ``build_osqp_plan`` 574-662).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from warpmpc_b200.jax_qdldl.planning import build_qdldl_plan

from .types import FixedOSQPPlan, OSQPDerivativePlan, OSQPSettings

OSQP_INFTY = 1e30
OSQP_MIN_SCALING = 1e-4
OSQP_MAX_SCALING = 1e4


@dataclass(frozen=True)
class _ScalingData:
    c: float
    cinv: float
    d: np.ndarray
    dinv: np.ndarray
    e: np.ndarray
    einv: np.ndarray
    p_scale: np.ndarray
    a_scale: np.ndarray
    q_scale: np.ndarray
    y_scale: np.ndarray
    y_unscale: np.ndarray


def _csc_rows_cols(matrix: sp.csc_matrix):
    """Row and column index of every stored entry, in storage order."""
    cols = np.repeat(np.arange(matrix.shape[1], dtype=np.int32), np.diff(matrix.indptr))
    return np.asarray(matrix.indices, dtype=np.int32), cols


def _upper_with_diagonal(matrix: sp.spmatrix) -> sp.csc_matrix:
    """Upper triangle of P; missing diagonal slots are requested explicitly.

    The request goes through SciPy's sparse addition exactly as in
    solver.py:64-78, so the resulting pattern is the same as the reference's
    (SciPy drops explicit zeros produced by the addition).
    """
    upper = sp.triu(matrix, format="csc")
    upper.sum_duplicates()
    upper.sort_indices()
    n = upper.shape[0]
    rows, cols = _csc_rows_cols(upper)
    has_diag = np.zeros(n, dtype=bool)
    has_diag[cols[rows == cols]] = True
    if not np.all(has_diag):
        missing = np.flatnonzero(~has_diag)
        filler = sp.csc_matrix((np.zeros_like(missing, dtype=float), (missing, missing)), shape=upper.shape)
        upper = (upper + filler).tocsc()
        upper.sum_duplicates()
        upper.sort_indices()
    return upper


def _build_kkt_and_maps(p_upper: sp.csc_matrix, a_matrix: sp.csc_matrix, settings: OSQPSettings, rho_inv_vec: np.ndarray):
    """KKT upper pattern and value maps (solver.py:81-150).

    KKT rows/cols: ``0..n-1`` primal, ``n..n+m-1`` constraints.  Entries are
    sorted column-major; ``p_to_kkt[k]``/``a_to_kkt[k]``/``rho_to_kkt[r]`` give
    the KKT storage slot of P entry ``k``, A entry ``k`` and constraint ``r``.
    """

    n = p_upper.shape[0]
    m = a_matrix.shape[0]
    p_rows, p_cols = _csc_rows_cols(p_upper)
    a_rows, a_cols = _csc_rows_cols(a_matrix)
    p_vals = np.asarray(p_upper.data, dtype=np.float64).copy()
    on_diag = p_rows == p_cols
    p_vals[on_diag] = p_vals[on_diag] + settings.sigma
    diag_present = np.zeros(n, dtype=bool)
    diag_present[p_cols[on_diag]] = True
    extra_diag = np.flatnonzero(~diag_present).astype(np.int32)

    # (row, col, value) of every KKT entry; group tags keep track of origin
    rows = np.concatenate([p_rows, extra_diag, a_cols, n + np.arange(m, dtype=np.int32)])
    cols = np.concatenate([p_cols, extra_diag, n + a_rows, n + np.arange(m, dtype=np.int32)])
    vals = np.concatenate(
        [
            p_vals,
            np.full(extra_diag.size, settings.sigma, dtype=np.float64),
            np.asarray(a_matrix.data, dtype=np.float64),
            -np.asarray(rho_inv_vec, dtype=np.float64),
        ]
    )
    order = np.lexsort((rows, cols))
    slot = np.empty(order.size, dtype=np.int64)
    slot[order] = np.arange(order.size)
    sorted_rows = rows[order]
    sorted_cols = cols[order]
    if np.any((np.diff(sorted_cols) == 0) & (np.diff(sorted_rows) == 0)):
        raise ValueError("duplicate KKT entry")
    kkt = sp.csc_matrix((vals[order], (sorted_rows, sorted_cols)), shape=(n + m, n + m))
    kkt.sum_duplicates()
    kkt.sort_indices()

    n_p = p_rows.size
    n_a = a_rows.size
    base = n_p + extra_diag.size
    p_to_kkt = slot[:n_p].astype(np.int32)
    a_to_kkt = slot[base : base + n_a].astype(np.int32)
    rho_to_kkt = slot[base + n_a :].astype(np.int32)
    p_diag_sigma = np.where(on_diag, settings.sigma, 0.0).astype(np.float64)
    return kkt, p_to_kkt, p_diag_sigma, a_to_kkt, rho_to_kkt


def _bounds_type(l: np.ndarray, u: np.ndarray) -> np.ndarray:
    """-1 loose (both infinite), 1 equality (|u-l| < 1e-4), 0 otherwise."""
    l = np.asarray(l, dtype=float)
    u = np.asarray(u, dtype=float)
    out = np.zeros(l.shape, dtype=np.int32)
    out[(l <= -OSQP_INFTY) & (u >= OSQP_INFTY)] = -1
    with np.errstate(invalid="ignore"):
        out[np.abs(u - l) < 1e-4] = 1
    return out


def _rho_vectors(settings: OSQPSettings, m: int, l, u):
    """Per-constraint rho (solver.py:164-183): 1e-6 loose, 1e3*rho equality."""
    if settings.rho_is_vec:
        if l is None or u is None:
            raise ValueError("l and u are required when settings.rho_is_vec=True")
        constr_type = _bounds_type(np.asarray(l)[:m], np.asarray(u)[:m])
        rho_vec = np.full(m, settings.rho, dtype=np.float64)
        rho_vec[constr_type < 0] = 1e-6
        rho_vec[constr_type > 0] = 1e3 * settings.rho
    else:
        constr_type = np.zeros(m, dtype=np.int32)
        rho_vec = np.full(m, settings.rho, dtype=np.float64)
    rho_vec = rho_vec.astype(np.float64)
    return rho_vec, 1.0 / rho_vec, constr_type


def _p_full_pattern(p_upper: sp.csc_matrix):
    """Both triangles of P as (row, col, upper-entry index) triples (solver.py:186-204)."""
    rows, cols = _csc_rows_cols(p_upper)
    idx = np.arange(rows.size, dtype=np.int32)
    off = rows != cols
    # entry k, then (if off-diagonal) its mirror, interleaved in storage order
    full_rows = np.empty(rows.size + int(off.sum()), dtype=np.int32)
    full_cols = np.empty_like(full_rows)
    full_map = np.empty_like(full_rows)
    mirrors_before = np.concatenate([[0], np.cumsum(off)[:-1]]).astype(np.int64) if rows.size else np.zeros(0, np.int64)
    pos = np.arange(rows.size, dtype=np.int64) + mirrors_before
    full_rows[pos] = rows
    full_cols[pos] = cols
    full_map[pos] = idx
    mirror_pos = pos[off] + 1
    full_rows[mirror_pos] = cols[off]
    full_cols[mirror_pos] = rows[off]
    full_map[mirror_pos] = idx[off]
    return full_rows, full_cols, full_map


def _col_inf_norm(matrix: sp.csc_matrix) -> np.ndarray:
    out = np.zeros(matrix.shape[1], dtype=np.float64)
    absval = np.abs(np.asarray(matrix.data, dtype=np.float64))
    _, cols = _csc_rows_cols(matrix)
    if absval.size:
        np.maximum.at(out, cols, absval)
    return out


def _row_inf_norm(matrix: sp.csc_matrix) -> np.ndarray:
    out = np.zeros(matrix.shape[0], dtype=np.float64)
    absval = np.abs(np.asarray(matrix.data, dtype=np.float64))
    if absval.size:
        np.maximum.at(out, np.asarray(matrix.indices), absval)
    return out


def _clip_scaling(values: np.ndarray) -> np.ndarray:
    values = np.asarray(values, dtype=np.float64).copy()
    values[values < OSQP_MIN_SCALING] = 1.0
    values[values > OSQP_MAX_SCALING] = OSQP_MAX_SCALING
    return values


def _clip_scaling_scalar(value: float) -> float:
    if value < OSQP_MIN_SCALING:
        return 1.0
    return float(min(value, OSQP_MAX_SCALING))


def _nominal_scaling_q(q, n: int):
    if q is None:
        return None
    q_array = np.asarray(q, dtype=np.float64)
    if q_array.ndim == 2 and q_array.shape[0] == 1:
        q_array = q_array[0]
    if q_array.shape != (n,):
        raise ValueError("scaling_q must have shape (n,) or (1, n)")
    return q_array.copy()


def _compute_scaling(p_upper: sp.csc_matrix, a_matrix: sp.csc_matrix, iterations: int, *, q=None) -> _ScalingData:
    """Ruiz equilibration with cost scaling (OSQP; solver.py:262-343).

    ``iterations`` rounds of D <- D / sqrt(col inf-norms of [P; A]) and
    E <- E / sqrt(row inf-norms of A), then the cost factor
    c <- c / clip(max(mean col norm of P, |q|_inf)).  Norms of P are taken
    over its stored upper triangle, as in the reference.
    """

    n = p_upper.shape[0]
    m = a_matrix.shape[0]
    d = np.ones(n, dtype=np.float64)
    e = np.ones(m, dtype=np.float64)
    c = 1.0
    p_rows, p_cols = _csc_rows_cols(p_upper)
    a_rows, a_cols = _csc_rows_cols(a_matrix)
    if iterations <= 0:
        return _ScalingData(
            c=1.0, cinv=1.0, d=d, dinv=d.copy(), e=e, einv=e.copy(),
            p_scale=np.ones(p_upper.nnz, dtype=np.float64),
            a_scale=np.ones(a_matrix.nnz, dtype=np.float64),
            q_scale=d.copy(), y_scale=e.copy(), y_unscale=e.copy(),
        )

    p_work = p_upper.copy().astype(np.float64)
    a_work = a_matrix.copy().astype(np.float64)
    q_work = _nominal_scaling_q(q, n)
    for _ in range(iterations):
        d_step = _clip_scaling(np.maximum(_col_inf_norm(p_work), _col_inf_norm(a_work)))
        e_step = _clip_scaling(_row_inf_norm(a_work))
        d_step = 1.0 / np.sqrt(d_step)
        e_step = 1.0 / np.sqrt(e_step)
        p_work.data *= d_step[p_rows] * d_step[p_cols]
        a_work.data *= e_step[a_rows] * d_step[a_cols]
        if q_work is not None:
            q_work *= d_step
        d *= d_step
        e *= e_step
        p_measure = float(np.sum(_col_inf_norm(p_work)) / n)
        q_measure = 0.0 if q_work is None else float(np.max(np.abs(q_work)))
        q_measure = _clip_scaling_scalar(q_measure)
        gamma = 1.0 / _clip_scaling_scalar(max(p_measure, q_measure))
        p_work.data *= gamma
        if q_work is not None:
            q_work *= gamma
        c *= gamma

    dinv = 1.0 / d
    einv = 1.0 / e
    cinv = 1.0 / c
    return _ScalingData(
        c=float(c), cinv=float(cinv), d=d, dinv=dinv, e=e, einv=einv,
        p_scale=c * d[p_rows] * d[p_cols],
        a_scale=e[a_rows] * d[a_cols],
        q_scale=c * d, y_scale=c * einv, y_unscale=cinv * e,
    )


def build_osqp_plan(
    p_matrix: sp.spmatrix,
    a_matrix: sp.spmatrix,
    l: np.ndarray | None = None,
    u: np.ndarray | None = None,
    settings: OSQPSettings | None = None,
    derivatives: bool = False,
    scaling_q: np.ndarray | None = None,
    *,
    perm: np.ndarray | None = None,
) -> FixedOSQPPlan:
    """All fixed-pattern OSQP direct-solver setup on the host (solver.py:574-662).

    ``perm`` optionally fixes the KKT ordering (default: AMD).
    """

    settings = OSQPSettings() if settings is None else settings
    if settings.scaling < 0:
        raise ValueError("settings.scaling must be nonnegative")
    if settings.adaptive_rho and (settings.adaptive_rho_interval < 1 or settings.adaptive_rho_tolerance < 1.0):
        raise ValueError("adaptive_rho needs adaptive_rho_interval >= 1 and adaptive_rho_tolerance >= 1")
    if settings.polishing:
        raise NotImplementedError("the fixed-pattern OSQP solver expects polishing=False")

    p_upper = _upper_with_diagonal(p_matrix)
    a_csc = sp.csc_matrix(a_matrix)
    a_csc.sum_duplicates()
    a_csc.sort_indices()
    if p_upper.shape[0] != p_upper.shape[1]:
        raise ValueError("P must be square")
    if a_csc.shape[1] != p_upper.shape[0]:
        raise ValueError("A column count must match P dimension")

    scaling = _compute_scaling(p_upper, a_csc, settings.scaling, q=scaling_q)
    scaled_l = None if l is None else np.asarray(l, dtype=np.float64) * scaling.e
    scaled_u = None if u is None else np.asarray(u, dtype=np.float64) * scaling.e
    rho_vec, rho_inv_vec, constr_type = _rho_vectors(settings, a_csc.shape[0], scaled_l, scaled_u)
    p_kkt = p_upper.copy()
    a_kkt = a_csc.copy()
    p_kkt.data = np.asarray(p_kkt.data, dtype=np.float64) * scaling.p_scale
    a_kkt.data = np.asarray(a_kkt.data, dtype=np.float64) * scaling.a_scale
    kkt, p_to_kkt, p_diag_sigma, a_to_kkt, rho_to_kkt = _build_kkt_and_maps(p_kkt, a_kkt, settings, rho_inv_vec)
    qdldl_plan = build_qdldl_plan(kkt, upper=True, perm=perm)
    p_rows, p_cols, p_value_map = _p_full_pattern(p_upper)
    derivative_plan = _build_derivative_plan(p_upper, a_csc, l, u) if derivatives else None
    a_rows, a_cols = _csc_rows_cols(a_csc)

    return FixedOSQPPlan(
        n=p_upper.shape[0],
        m=a_csc.shape[0],
        p_upper=p_upper,
        a_matrix=a_csc,
        kkt_upper=kkt,
        qdldl_plan=qdldl_plan,
        p_to_kkt=p_to_kkt,
        p_diag_sigma=p_diag_sigma,
        a_to_kkt=a_to_kkt,
        rho_to_kkt=rho_to_kkt,
        a_rows=a_rows,
        a_cols=a_cols,
        p_full_rows=p_rows,
        p_full_cols=p_cols,
        p_full_value_map=p_value_map,
        rho_vec=rho_vec,
        rho_inv_vec=rho_inv_vec,
        constr_type=constr_type,
        scaling_c=scaling.c,
        scaling_cinv=scaling.cinv,
        scaling_d=scaling.d,
        scaling_dinv=scaling.dinv,
        scaling_e=scaling.e,
        scaling_einv=scaling.einv,
        p_scale=scaling.p_scale,
        a_scale=scaling.a_scale,
        q_scale=scaling.q_scale,
        y_scale=scaling.y_scale,
        y_unscale=scaling.y_unscale,
        derivative_plan=derivative_plan,
        settings=settings,
    )


def _build_derivative_plan(p_upper, a_matrix, l, u):
    """Reference-style adjoint KKT plan; defined in :mod:`.derivative_plan`."""
    from .derivative_plan import build_derivative_plan

    return build_derivative_plan(p_upper, a_matrix, l, u)
