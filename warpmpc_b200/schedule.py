"""Host view of the streaming schedule built by the C library.

``stream_schedule(osqp_plan)`` returns the chunk tables, meta blocks, stream
positions, release order and compact-accumulator tables the persistent
streaming kernel uses for a plan (``wmpc_stream_schedule_host``; no GPU
needed).  Used to inspect and verify the schedule on the CPU.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import native
from .jax_qdldl.planning import plan_ragged_program

DEFAULT_TARGETS = (24, 24, 16, 24, 0)  # backward units, columns, releases; forward units; offload bits (the library's)


def _pattern_desc(qp):
    rg = plan_ragged_program(qp)
    arrays = {
        "perm_to_orig": native.i32(qp.perm_to_orig),
        "diag_pos": native.i32(qp.diag_pos),
        "init_ptr": native.i32(rg["init_ptr"]),
        "init_rows": native.i32(rg["init_rows"]),
        "init_pos": native.i32(rg["init_pos"]),
        "proc_ptr": native.i32(rg["proc_ptr"]),
        "proc_cols": native.i32(rg["proc_cols"]),
        "proc_lidx": native.i32(rg["proc_lidx"]),
        "proc_offsets": native.i32(rg["proc_offsets"]),
        "lp": native.i32(qp.lp),
        "li": native.i32(qp.li),
        "p": native.i32(qp.p),
        "pinv": native.i32(qp.pinv),
    }
    desc = native.PatternDesc(n=qp.n, nnz_a=qp.nnz_a, nnz_l=qp.nnz_l,
                              **{k: native.ptr_i32(v) for k, v in arrays.items()})
    return desc, arrays, rg


def solve_tables(qdldl_plan) -> dict:
    """Chunk tables of the TMA-fed per-call solve for a QDLDL plan
    (``wmpc_solve_tables_host``): ``tables`` (int32 words) and ``desc``
    (n_chunks x 8: table word offset, words, e0, c0, entries, columns, 0, 0)."""
    desc, keep, _ = _pattern_desc(qdldl_plan)
    lib = native.lib()
    words = ctypes.c_int64()
    native.check(lib.wmpc_solve_tables_host(ctypes.byref(desc), None, 0, ctypes.byref(words)))
    buf = np.empty(words.value, dtype=np.int32)
    native.check(lib.wmpc_solve_tables_host(ctypes.byref(desc), native.ptr_i32(buf), buf.size, ctypes.byref(words)))
    n_chunks, tw = int(buf[0]), int(buf[1])
    return {"tables": buf[2 : 2 + tw].copy(), "desc": buf[2 + tw : 2 + tw + 8 * n_chunks].reshape(n_chunks, 8).copy()}


def stream_schedule(plan, targets=DEFAULT_TARGETS) -> dict:
    """Schedule of an OSQP plan (rho per constraint) as NumPy arrays.

    targets: (backward units, backward columns, backward releases, forward
    units) per chunk, and the offload bits (1: leaf columns, 2: rows reading
    only leaf rows, solved by the releasing warp; 4: the frontier-slot form)."""
    qp = plan.qdldl_plan
    desc, keep, rg = _pattern_desc(qp)
    rho = native.f32(plan.rho_vec)
    rinv = native.f32(plan.rho_inv_vec)
    lib = native.lib()
    words = ctypes.c_int64()
    args = (ctypes.byref(desc), native.ptr_f32(rho), native.ptr_f32(rinv), int(plan.n), *map(int, targets))
    native.check(lib.wmpc_stream_schedule_host(*args, None, 0, ctypes.byref(words)))
    buf = np.empty(words.value, dtype=np.int32)
    native.check(lib.wmpc_stream_schedule_host(*args, native.ptr_i32(buf), buf.size, ctypes.byref(words)))
    n, nnz_l = qp.n, qp.nnz_l
    hdr = buf[:8]
    n_chunks, blen, max_units, max_cols, max_rel, max_meta, max_row, n_meta = (int(v) for v in hdr)
    pos = 8
    out = {"n_chunks": n_chunks, "blen": blen, "max_units": max_units, "max_cols": max_cols,
           "max_rel": max_rel, "max_meta_words": max_meta, "max_row_nnz": max_row}

    def take(name, count):
        nonlocal pos
        out[name] = buf[pos : pos + count].copy()
        pos += count

    take("chunk_off", n_chunks + 1)
    take("chunk_units", n_chunks)
    take("chunk_cols", n_chunks)
    take("chunk_u0", n_chunks)
    take("chunk_nrel", n_chunks)
    take("meta_off", n_chunks)
    take("meta_words", n_chunks)
    take("meta", n_meta)
    take("col_uoff", n)
    take("dinv_off", n)
    take("proc_boff", nnz_l)
    take("u_perm", n)
    take("u_orig", n)
    take("init_slot", int(rg["init_ptr"][-1]))
    take("upd_ptr", nnz_l + 1)
    take("upd_slot", int(out["upd_ptr"][-1]))
    nf, flen, mfu, mfm, nfm = (int(v) for v in buf[pos : pos + 5])
    pos += 5
    out.update({"n_fchunks": nf, "flen": flen, "max_funits": mfu, "max_fmeta_words": mfm})
    take("fchunk_off", nf + 1)
    take("fchunk_units", nf)
    take("fmeta_off", nf)
    take("fmeta_words", nf)
    take("fmeta", nfm)
    take("proc_foff", nnz_l)
    npb, npf, ndum = (int(v) for v in buf[pos : pos + 3])
    pos += 3
    out["dummy_units"] = ndum
    take("pad_boff", npb)
    take("pad_foff", npf)
    take("chunk_pre_u0", n_chunks)
    take("chunk_pre_units", n_chunks)
    fs, flag, mfr = (int(v) for v in buf[pos : pos + 3])
    pos += 3
    out.update({"frontier_slots": fs, "frontier_lag": flag, "max_frows": mfr})
    assert pos == buf.size
    out["ragged"] = rg
    return out
