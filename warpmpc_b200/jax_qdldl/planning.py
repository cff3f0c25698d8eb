"""Host-side symbolic analysis for the fixed-pattern batched LDL^T path.

Everything here runs once per sparsity pattern on the host and produces the
integer tables the CUDA kernels consume.  Each function reproduces the output
of the reference function named in its docstring exactly (same arrays, same
dtypes, same entry order), because the tables define the floating-point
operation order of the factorization and solves; parity tests compare them
array-for-array with the reference.  The implementations are this project's
own (vectorised NumPy where the algorithm allows it).

Reference: ``warpmpc/jax_qdldl/core.py`` (``_as_upper_csc`` 38-46,
``_symperm_upper`` 55-102, ``_qdldl_etree`` 105-131, ``_build_numeric_program``
147-256, ``build_qdldl_plan`` 259-311, segmentation 320-485,
``_make_solve_levels`` 488-510) and ``warpmpc/jax_qdldl/warp_backend.py``
(``_pack_levels`` 1098-1104, ``_make_level_schedule`` 1107-1126,
``_make_segment_arrays`` 1129-1149).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .amd import amd_order
from .types import QDLDLPlan

QDLDL_UNKNOWN = -1


def _as_upper_csc(matrix: sp.spmatrix, upper: bool) -> sp.csc_matrix:
    """Upper-triangular CSC with summed duplicates and sorted rows (core.py:38-46)."""
    matrix = sp.csc_matrix(matrix)
    out = matrix.copy() if upper else sp.triu(matrix, format="csc")
    out.sum_duplicates()
    out.sort_indices()
    return out


def _pinv(p: np.ndarray) -> np.ndarray:
    inv = np.empty_like(p)
    inv[p] = np.arange(p.size, dtype=p.dtype)
    return inv


def _symperm_upper(matrix: sp.csc_matrix, pinv: np.ndarray):
    """Symmetric permutation ``P A P^T`` of an upper CSC matrix (core.py:55-102).

    Entries are placed into permuted column ``max(pinv[i], pinv[j])`` in the
    order in which they appear in the input (column-major, then stored order),
    which a stable sort by destination column reproduces.  Returns
    ``(cp int32, ci int32, cx, orig_to_perm int32)``.
    """

    n = matrix.shape[0]
    ap = np.asarray(matrix.indptr)
    ai = np.asarray(matrix.indices)
    ax = np.asarray(matrix.data)
    col_of = np.repeat(np.arange(n, dtype=np.int64), np.diff(ap))
    keep = ai <= col_of
    kept = np.flatnonzero(keep)
    i2 = np.asarray(pinv, dtype=np.int64)[ai[kept]]
    j2 = np.asarray(pinv, dtype=np.int64)[col_of[kept]]
    dest_col = np.maximum(i2, j2)
    dest_row = np.minimum(i2, j2)
    order = np.argsort(dest_col, kind="stable")
    cp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(dest_col, minlength=n), out=cp[1:])
    ci = dest_row[order].astype(np.int32)
    cx = ax[kept][order]
    orig_to_perm = np.full(ap[-1], -1, dtype=np.int32)
    orig_to_perm[kept[order]] = np.arange(order.size, dtype=np.int32)
    if np.any(orig_to_perm < 0):
        raise ValueError("input matrix contains lower-triangular entries")
    return cp.astype(np.int32), ci, cx, orig_to_perm


def _qdldl_etree(n: int, ap: np.ndarray, ai: np.ndarray):
    """Elimination tree and column counts of L (QDLDL_etree; core.py:105-131).

    Returns ``(lnz int32, etree int32, nnz_l)``; ``etree[i] = -1`` marks a root.
    """

    ap = np.asarray(ap)
    ai = np.asarray(ai)
    empty = np.flatnonzero(ap[1:] == ap[:-1])
    if empty.size:
        raise ValueError(f"column {int(empty[0])} is empty; QDLDL requires a nonempty column")
    visited_by = np.zeros(n, dtype=np.int32)
    counts = np.zeros(n, dtype=np.int32)
    parent = np.full(n, QDLDL_UNKNOWN, dtype=np.int32)
    ai_list = ai.tolist()
    ap_list = ap.tolist()
    for j in range(n):
        visited_by[j] = j
        for i in ai_list[ap_list[j] : ap_list[j + 1]]:
            if i > j:
                raise ValueError("matrix is not upper triangular after permutation")
            # climb from row i towards j, counting one L entry per new node
            while visited_by[i] != j:
                if parent[i] == QDLDL_UNKNOWN:
                    parent[i] = j
                counts[i] += 1
                visited_by[i] = j
                i = int(parent[i])
    return counts, parent, int(np.sum(counts, dtype=np.int64))


def _ragged_to_padded(ptr: np.ndarray, flat: np.ndarray):
    """Pad ragged rows to a dense ``(rows, max_len)`` int32 array plus bool mask."""
    lengths = np.diff(ptr)
    rows = lengths.size
    width = int(lengths.max()) if rows else 0
    out = np.zeros((rows, width), dtype=np.int32)
    mask = np.zeros((rows, width), dtype=bool)
    if width and flat.size:
        row_of = np.repeat(np.arange(rows), lengths)
        col_of = np.arange(flat.size) - np.repeat(ptr[:-1], lengths)
        out[row_of, col_of] = flat
        mask[row_of, col_of] = True
    return out, mask


def _numeric_program_ragged(n: int, ap: np.ndarray, ai: np.ndarray, lnz: np.ndarray, etree: np.ndarray):
    """Row-by-row program of the up-looking QDLDL factorization, ragged form.

    For row ``k``: ``init`` lists the off-diagonal entries of permuted column
    ``k`` (rows and positions, stored order), and ``proc`` lists the columns
    ``cidx`` of row ``k`` of L in the order the factorization visits them (the
    reverse of the etree-reach order), with the L slot each one fills and its
    offset inside its column.  Same content as core.py:147-256.
    """

    lp = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(lnz, out=lp[1:])
    nnz_l = int(lp[-1])
    li = np.empty(nnz_l, dtype=np.int32)
    fill = lp[:-1].astype(np.int64).copy()

    ap_list = np.asarray(ap).tolist()
    ai_list = np.asarray(ai).tolist()
    parent = np.asarray(etree).tolist()

    diag_pos = np.full(n, -1, dtype=np.int32)
    init_rows: list[int] = []
    init_pos: list[int] = []
    init_ptr = [0]
    proc_cols: list[int] = []
    proc_lidx: list[int] = []
    proc_off: list[int] = []
    proc_ptr = [0]
    mark = [-1] * n  # mark[i] == k  <=>  i already in the reach of row k

    for k in range(n):
        start, stop = ap_list[k], ap_list[k + 1]
        reach: list[int] = []
        for ptr in range(start, stop):
            row = ai_list[ptr]
            if row == k:
                diag_pos[k] = ptr
                continue
            init_rows.append(row)
            init_pos.append(ptr)
            if k == 0 or mark[row] == k:
                continue
            # walk up the etree until a marked node, k, or a root
            path = [row]
            mark[row] = k
            node = parent[row]
            while node != QDLDL_UNKNOWN and node < k and mark[node] != k:
                mark[node] = k
                path.append(node)
                node = parent[node]
            path.reverse()
            reach.extend(path)
        if diag_pos[k] < 0:
            raise ValueError(f"column {k} has no diagonal entry")
        init_ptr.append(len(init_rows))
        for cidx in reversed(reach):
            slot = int(fill[cidx])
            proc_cols.append(cidx)
            proc_lidx.append(slot)
            proc_off.append(slot - int(lp[cidx]))
            li[slot] = k
            fill[cidx] = slot + 1
        proc_ptr.append(len(proc_cols))

    if not np.array_equal(fill, lp[1:]):
        raise AssertionError("internal symbolic program did not fill L correctly")

    as32 = lambda v: np.asarray(v, dtype=np.int32)  # noqa: E731
    return {
        "lp": lp,
        "li": li,
        "diag_pos": diag_pos,
        "init_ptr": as32(init_ptr),
        "init_rows": as32(init_rows),
        "init_pos": as32(init_pos),
        "proc_ptr": as32(proc_ptr),
        "proc_cols": as32(proc_cols),
        "proc_lidx": as32(proc_lidx),
        "proc_offsets": as32(proc_off),
    }


def _build_numeric_program(n: int, ap: np.ndarray, ai: np.ndarray, lnz: np.ndarray, etree: np.ndarray):
    """Padded numeric program with the reference's keys (core.py:147-256)."""

    rg = _numeric_program_ragged(n, ap, ai, lnz, etree)
    init_rows, init_mask = _ragged_to_padded(rg["init_ptr"], rg["init_rows"])
    init_pos, _ = _ragged_to_padded(rg["init_ptr"], rg["init_pos"])
    process_cols, process_mask = _ragged_to_padded(rg["proc_ptr"], rg["proc_cols"])
    process_lidx, _ = _ragged_to_padded(rg["proc_ptr"], rg["proc_lidx"])
    process_offsets, _ = _ragged_to_padded(rg["proc_ptr"], rg["proc_offsets"])
    lp = rg["lp"]
    col_rows, col_mask = _ragged_to_padded(lp, rg["li"])
    col_lidx, _ = _ragged_to_padded(lp, np.arange(lp[-1], dtype=np.int32))
    return {
        "lp": lp,
        "li": rg["li"],
        "diag_pos": rg["diag_pos"],
        "init_rows": init_rows,
        "init_pos": init_pos,
        "init_mask": init_mask,
        "process_cols": process_cols,
        "process_lidx": process_lidx,
        "process_offsets": process_offsets,
        "process_mask": process_mask,
        "col_rows": col_rows,
        "col_lidx": col_lidx,
        "col_mask": col_mask,
    }


def build_qdldl_plan(
    matrix: sp.spmatrix,
    upper: bool = False,
    *,
    perm: np.ndarray | None = None,
) -> QDLDLPlan:
    """Build a fixed-pattern plan from a symmetric matrix (core.py:259-311).

    ``perm`` (new index -> old index) overrides the AMD ordering; by default
    the ordering is :func:`warpmpc_b200.jax_qdldl.amd.amd_order`.
    """

    a_upper = _as_upper_csc(matrix, upper=upper)
    n = a_upper.shape[0]
    if a_upper.shape[0] != a_upper.shape[1]:
        raise ValueError("QDLDL matrix must be square")
    p = amd_order(a_upper) if perm is None else np.asarray(perm)
    p = np.asarray(p, dtype=np.int32)
    if p.shape != (n,) or not np.array_equal(np.sort(p), np.arange(n)):
        raise ValueError("perm must be a permutation of range(n)")
    pinv = _pinv(p)
    aperm_p, aperm_i, _, orig_to_perm = _symperm_upper(a_upper, pinv)
    perm_to_orig = np.empty_like(orig_to_perm)
    perm_to_orig[orig_to_perm] = np.arange(orig_to_perm.size, dtype=np.int32)
    lnz, etree, nnz_l = _qdldl_etree(n, aperm_p, aperm_i)
    program = _build_numeric_program(n, aperm_p, aperm_i, lnz, etree)
    return QDLDLPlan(
        n=n,
        nnz_a=int(a_upper.indptr[-1]),
        nnz_l=nnz_l,
        a_indptr=np.asarray(a_upper.indptr, dtype=np.int32),
        a_indices=np.asarray(a_upper.indices, dtype=np.int32),
        a_data=np.asarray(a_upper.data),
        aperm_indptr=aperm_p,
        aperm_indices=aperm_i,
        perm_to_orig=perm_to_orig,
        orig_to_perm=orig_to_perm,
        p=p,
        pinv=pinv,
        etree=etree,
        lnz=lnz,
        **program,
    )


def plan_ragged_program(plan: QDLDLPlan) -> dict[str, np.ndarray]:
    """Ragged (CSR-style) form of a plan's row program, as the kernels use it."""
    return _numeric_program_ragged(plan.n, plan.aperm_indptr, plan.aperm_indices, plan.lnz, plan.etree)


# ---------------------------------------------------------------------------
# segmentation of padded loops (core.py:320-485; warp_backend.py:1129-1149)
# ---------------------------------------------------------------------------


def _row_counts(mask: np.ndarray) -> np.ndarray:
    return np.asarray(np.sum(mask, axis=1), dtype=np.int64)


def _as_segments(intervals) -> list[tuple[int, np.ndarray]]:
    return [(int(a), np.arange(a, b, dtype=np.int32)) for a, b in intervals]


def _check_budget(segment_budget: int) -> None:
    if segment_budget <= 0:
        raise ValueError("segment_budget must be positive")


def _make_fixed_segments(mask: np.ndarray, segment_budget: int):
    """``min(budget, n)`` nearly equal contiguous segments (core.py:347-360)."""
    n = int(mask.shape[0])
    if n == 0:
        return []
    _check_budget(segment_budget)
    edges = np.linspace(0, n, min(int(segment_budget), n) + 1, dtype=np.int64)
    return _as_segments(zip(edges[:-1], edges[1:]))


def _split_saving(counts: np.ndarray, start: int, stop: int):
    """Best single split of ``[start, stop)`` and the padded work it saves."""
    length = stop - start
    if length <= 1:
        return None, 0
    seg = counts[start:stop]
    whole = length * int(seg.max(initial=0))
    prefix_max = np.maximum.accumulate(seg)[:-1]
    suffix_max = np.maximum.accumulate(seg[::-1])[::-1][1:]
    cut = np.arange(1, length, dtype=np.int64)
    saving = whole - cut * prefix_max - (length - cut) * suffix_max
    best = int(np.argmax(saving))
    if saving[best] <= 0:
        return None, 0
    return start + best + 1, int(saving[best])


def _make_adaptive_segments(mask: np.ndarray, segment_budget: int):
    """Greedy splitting by largest padded-work saving (core.py:363-396)."""
    n = int(mask.shape[0])
    if n == 0:
        return []
    _check_budget(segment_budget)
    counts = _row_counts(mask)
    intervals = [(0, n)]
    target = min(int(segment_budget), n)
    while len(intervals) < target:
        choice = None
        best = 0
        for idx, (a, b) in enumerate(intervals):
            cut, saving = _split_saving(counts, a, b)
            if saving > best:
                choice, best = (idx, cut), saving
        if choice is None:
            break
        idx, cut = choice
        a, b = intervals[idx]
        intervals[idx : idx + 1] = [(a, cut), (cut, b)]
    return _as_segments(intervals)


def _make_optimal_segments(mask: np.ndarray, segment_budget: int):
    """Exactly ``min(budget, n)`` contiguous segments of minimum padded work.

    ``cost[k][j] = min_i cost[k-1][i] + (j - i) * max(counts[i:j])``; among
    equal costs the smallest start ``i`` is kept, which is the choice the
    reference's grouped dynamic program makes (core.py:399-470).  Solved here
    as a dense vectorised DP over all (start, end) pairs.
    """

    n = int(mask.shape[0])
    if n == 0:
        return []
    _check_budget(segment_budget)
    target = min(int(segment_budget), n)
    counts = _row_counts(mask)
    big = np.int64(1) << np.int64(62)
    # seg_cost[j, i] = (j - i) * max(counts[i:j]) for i < j, else "infinite"
    seg_cost = np.full((n + 1, n + 1), big, dtype=np.int64)
    for j in range(1, n + 1):
        suffix_max = np.maximum.accumulate(counts[:j][::-1])[::-1]
        seg_cost[j, :j] = (j - np.arange(j, dtype=np.int64)) * suffix_max
    prev = np.full(n + 1, big, dtype=np.int64)
    prev[0] = 0
    back = np.full((target + 1, n + 1), -1, dtype=np.int64)
    for k in range(1, target + 1):
        total = np.where(prev[None, :] >= big, big, prev[None, :] + seg_cost)
        total = np.minimum(total, big)
        arg = np.argmin(total, axis=1)
        best = total[np.arange(n + 1), arg]
        cur = np.where(best >= big, big, best)
        valid = (np.arange(n + 1) >= k) & (best < big)
        back[k, valid] = arg[valid]
        cur[~valid] = big
        prev = cur
    intervals = []
    end = n
    for k in range(target, 0, -1):
        start = int(back[k, end])
        if start < 0:
            raise AssertionError("optimal segmentation backtracking failed")
        intervals.append((start, end))
        end = start
    if end != 0:
        raise AssertionError("optimal segmentation did not cover all columns")
    intervals.reverse()
    return _as_segments(intervals)


def _make_segments(mask: np.ndarray, *, segment_budget: int, segment_strategy: str = "optimal"):
    if segment_strategy == "fixed":
        return _make_fixed_segments(mask, segment_budget)
    if segment_strategy == "greedy":
        return _make_adaptive_segments(mask, segment_budget)
    if segment_strategy == "optimal":
        return _make_optimal_segments(mask, segment_budget)
    raise ValueError(f"unknown segment_strategy {segment_strategy!r}")


def _make_segment_arrays(mask: np.ndarray, *, segment_budget: int, segment_strategy: str):
    """Segment starts, lengths and padded widths as int32 arrays."""
    segments = _make_segments(mask, segment_budget=segment_budget, segment_strategy=segment_strategy)
    counts_per_row = np.asarray(np.sum(mask, axis=1), dtype=np.int64) if mask.size else np.zeros(mask.shape[0], np.int64)
    starts = np.asarray([s for s, _ in segments], dtype=np.int32)
    lengths = np.asarray([c.size for _, c in segments], dtype=np.int32)
    widths = np.asarray([int(counts_per_row[c].max(initial=0)) for _, c in segments], dtype=np.int32)
    return starts, lengths, widths


# ---------------------------------------------------------------------------
# dependency levels of the triangular solves (core.py:488-510;
# warp_backend.py:1098-1126)
# ---------------------------------------------------------------------------


def _levels_from_csc(n: int, lp: np.ndarray, li: np.ndarray) -> np.ndarray:
    """Level of every column: 1 + max level of the columns it depends on."""
    level = np.zeros(n, dtype=np.int32)
    for col in range(n):
        rows = li[lp[col] : lp[col + 1]]
        if rows.size:
            np.maximum.at(level, rows, level[col] + 1)
    return level


def _make_solve_levels(col_rows: np.ndarray, col_mask: np.ndarray) -> list[np.ndarray]:
    """Columns grouped by dependency level, ascending (core.py:488-510)."""
    n = int(col_rows.shape[0])
    lengths = np.asarray(np.sum(col_mask, axis=1), dtype=np.int64) if col_mask.size else np.zeros(n, np.int64)
    lp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lengths, out=lp[1:])
    li = col_rows[np.asarray(col_mask, dtype=bool)] if col_mask.size else np.zeros(0, np.int32)
    level = _levels_from_csc(n, lp, li)
    top = int(level.max(initial=0))
    return [np.flatnonzero(level == lv).astype(np.int32) for lv in range(top + 1)]


def _pack_levels(levels):
    flat = np.concatenate([np.asarray(lv, dtype=np.int32) for lv in levels]) if levels else np.zeros(0, np.int32)
    offsets = np.zeros(len(levels) + 1, dtype=np.int32)
    np.cumsum([len(lv) for lv in levels], out=offsets[1:])
    return flat.astype(np.int32), offsets


def _make_level_schedule(levels, offsets, *, serial_width_threshold: int):
    """Runs of narrow levels become serial items; wide levels parallel items."""
    widths = [int(len(lv)) for lv in levels]
    schedule = []
    level = 0
    while level < len(widths):
        if widths[level] <= serial_width_threshold:
            first = level
            while level < len(widths) and widths[level] <= serial_width_threshold:
                level += 1
            schedule.append(("serial", first, level, int(offsets[first]), 0))
        else:
            schedule.append(("parallel", level, level + 1, int(offsets[level]), widths[level]))
            level += 1
    return tuple(schedule)
