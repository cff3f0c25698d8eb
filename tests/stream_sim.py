"""NumPy replay of the streaming persistent kernel (test helper).

Executes, for one tile of 32 instances, exactly the item sequence, meta
parsing, stream addressing and per-lane arithmetic of
``warpmpc_b200/csrc/persistent.cu`` (factor_stream_kernel,
state_to_stream_kernel, admm_stream_kernel, stream_to_state_kernel), with
bounds checks on every index, so the schedule and the kernel's index
arithmetic are verified on the CPU against the oracle.
"""

from __future__ import annotations

import numpy as np

KMETA = 5


def _f32(x):
    return np.float32(x)


def replay(plan, sched, p_values, a_values, q, l, u, x0=None, z0=None, y0=None, max_iter=None):
    """Run the stream algorithm for a batch of <= 32 instances (float32)."""
    qp = plan.qdldl_plan
    rg = sched["ragged"]
    n, nnz_l = qp.n, qp.nnz_l
    S = sched["stream_len"]
    B = q.shape[0]
    assert B <= 32
    lanes = 32
    pick = lambda arr: arr[np.minimum(np.arange(lanes), B - 1)]  # noqa: E731  (padding lanes copy the last)
    P = pick(np.atleast_2d(p_values) if np.atleast_2d(p_values).shape[0] > 1 else np.repeat(np.atleast_2d(p_values), B, 0))
    A = pick(np.atleast_2d(a_values) if np.atleast_2d(a_values).shape[0] > 1 else np.repeat(np.atleast_2d(a_values), B, 0))
    # KKT values (assemble_kkt_values), lanes x nnz_kkt
    kkt = np.broadcast_to(plan.kkt_upper.data.astype(np.float32), (lanes, plan.nnz_kkt)).copy()
    kkt[:, plan.p_to_kkt] = P * plan.p_scale.astype(np.float32) + plan.p_diag_sigma.astype(np.float32)
    kkt[:, plan.a_to_kkt] = A * plan.a_scale.astype(np.float32)
    # ---- factor_stream_kernel
    L = np.full((S, lanes), np.nan, dtype=np.float32)
    F = np.full((nnz_l, lanes), np.nan, dtype=np.float32)
    max_row = sched["max_row_nnz"]
    for k in range(n):
        p0, p1 = rg["proc_ptr"][k], rg["proc_ptr"][k + 1]
        assert p1 - p0 <= max_row
        ys = np.zeros((max(max_row, 1), lanes), dtype=np.float32)
        dk = kkt[:, qp.perm_to_orig[qp.diag_pos[k]]].copy()
        for e in range(rg["init_ptr"][k], rg["init_ptr"][k + 1]):
            s = sched["init_slot"][e]
            assert 0 <= s < p1 - p0
            ys[s] = ys[s] + kkt[:, qp.perm_to_orig[rg["init_pos"][e]]]
        for e in range(p0, p1):
            c = rg["proc_cols"][e]
            off = rg["proc_offsets"][e]
            base = sched["col_spos"][c]
            u0 = sched["upd_ptr"][e]
            val = ys[e - p0].copy()
            for qq in range(off):
                s = sched["upd_slot"][u0 + qq]
                assert 0 <= s < p1 - p0 and 0 <= base + qq < S and not np.isnan(L[base + qq]).any()
                ys[s] = ys[s] - L[base + qq] * val
            dpos = sched["dinv_spos"][c]
            assert not np.isnan(L[dpos]).any()
            lval = val * L[dpos]
            wpos = sched["proc_spos"][e]
            assert 0 <= wpos < S
            L[wpos] = lval
            fpos = sched["proc_fpos"][e]
            assert 0 <= fpos < nnz_l
            F[fpos] = lval
            dk = dk - val * lval
        L[sched["dinv_spos"][k]] = _f32(1.0) / dk
    assert not np.isnan(L).any(), "stream positions not all written"
    assert not np.isnan(F).any(), "forward stream positions not all written"
    # ---- state_to_stream_kernel (scaled)
    e_s = plan.scaling_e.astype(np.float32)
    qs = pick(q) * plan.q_scale.astype(np.float32)
    ls = pick(l) * e_s
    us = pick(u) * e_s
    xs = pick(x0) * plan.scaling_dinv.astype(np.float32) if x0 is not None else np.zeros((lanes, plan.n), np.float32)
    zs = pick(z0) * e_s if z0 is not None else np.zeros((lanes, plan.m), np.float32)
    ysc = pick(y0) * plan.y_scale.astype(np.float32) if y0 is not None else np.zeros((lanes, plan.m), np.float32)
    s0 = np.zeros((n, lanes), np.float32)
    s1 = np.zeros((n, lanes), np.float32)
    pp0 = np.zeros((n, lanes), np.float32)
    pp1 = np.zeros((n, lanes), np.float32)
    for uu in range(n):
        o = sched["u_orig"][uu]
        if o < plan.n:
            s0[uu], pp0[uu] = xs[:, o], qs[:, o]
        else:
            r = o - plan.n
            s0[uu], s1[uu], pp0[uu], pp1[uu] = zs[:, r], ysc[:, r], ls[:, r], us[:, r]
    # ---- admm_stream_kernel
    sigma = _f32(plan.settings.sigma)
    alpha = _f32(plan.settings.alpha)
    oma = _f32(1.0) - alpha
    iters = plan.settings.max_iter if max_iter is None else max_iter
    nch = sched["n_chunks"]
    X = np.full((n, lanes), np.nan, dtype=np.float32)
    meta_all = sched["meta"]

    def meta_of(ch):
        off, words = sched["meta_off"][ch], sched["meta_words"][ch]
        assert words <= sched["max_meta_words"] and off + words <= meta_all.size and words % 4 == 0
        return meta_all[off : off + words]

    nfc = sched["n_fchunks"]
    fmeta_all = sched["fmeta"]
    items = [(0, nch - 1 - t) for t in range(nch)]
    for _ in range(iters):
        items += [(1, c) for c in range(nfc)] + [(2, c) for c in range(nch - 1, -1, -1)]
    for kind, ch in items:
        if kind == 1:
            off, words = sched["fmeta_off"][ch], sched["fmeta_words"][ch]
            assert words <= sched["max_fmeta_words"] and words % 4 == 0 and off + words <= fmeta_all.size
            fm = fmeta_all[off : off + words]
            nrows, nent, r0 = int(fm[0]), int(fm[1]), int(fm[2])
            assert nent <= sched["max_fent"] and nrows <= sched["max_frows"]
            row_start = fm[4 : 4 + nrows + 1]
            coloff = fm[4 + nrows + 1 : 4 + nrows + 1 + nent]
            assert 4 + nrows + 1 + nent <= fm.size and np.all(coloff % 32 == 0)
            pos0 = sched["fchunk_pos"][ch]
            assert pos0 + nent <= nnz_l and sched["fchunk_pos"][ch + 1] - pos0 == nent
            Fs = F[pos0 : pos0 + nent]
            for i in range(nrows):
                acc = X[r0 + i].copy()
                for e in range(row_start[i], row_start[i + 1]):
                    c = coloff[e] // 32
                    assert 0 <= c < r0 + i
                    acc = acc - Fs[e] * X[c]
                X[r0 + i] = acc
            continue
        m = meta_of(ch)
        ncols, nent, nrel, c0, u0 = (int(v) for v in m[:KMETA])
        assert ncols == sched["chunk_cols"][ch] and nent == sched["chunk_ent"][ch]
        assert nent <= sched["max_ent"] and ncols <= sched["max_cols"] and nrel <= sched["max_rel"]
        col_start = m[KMETA : KMETA + ncols + 1]
        rows = m[KMETA + ncols + 1 : KMETA + ncols + 1 + nent]
        assert np.all(rows % 32 == 0)
        rows = rows // 32
        rel_i = m[KMETA + ncols + 1 + nent : KMETA + ncols + 1 + nent + nrel]
        rel_kind = m[KMETA + ncols + 1 + nent + nrel : KMETA + ncols + 1 + nent + 2 * nrel]
        rel_rho = m[KMETA + ncols + 1 + nent + 2 * nrel : KMETA + ncols + 1 + nent + 3 * nrel].view(np.float32)
        rel_rinv = m[KMETA + ncols + 1 + nent + 3 * nrel : KMETA + ncols + 1 + nent + 4 * nrel].view(np.float32)
        assert KMETA + ncols + 1 + nent + 4 * nrel <= m.size
        pos0 = sched["chunk_pos"][ch]
        count = nent if kind == 1 else nent + ncols if kind == 2 else 0
        assert pos0 + count <= S
        Ls = L[pos0 : pos0 + count]
        if kind == 1:
            for j in range(ncols):
                e0, e1 = col_start[j], col_start[j + 1]
                val = X[c0 + j].copy()
                for e in range(e0, e1):
                    r = rows[e]
                    assert 0 <= r < n
                    X[r] = X[r] - Ls[e] * val
        elif kind == 2:
            assert 0 <= u0 and u0 + nrel <= n
            for j in range(ncols - 1, -1, -1):
                e0, e1 = col_start[j], col_start[j + 1]
                corr = np.zeros(lanes, np.float32)
                for e in range(e0, e1):
                    corr = corr + Ls[e] * X[rows[e]]
                X[c0 + j] = X[c0 + j] * Ls[nent + j] - corr
            for k in range(nrel):
                i = rel_i[k]
                uu = u0 + k
                sol = X[i].copy()
                if rel_kind[k] == 0:
                    xn = alpha * sol + oma * s0[uu]
                    s0[uu] = xn
                    X[i] = sigma * xn - pp0[uu]
                else:
                    rinv = rel_rinv[k]
                    zk, yk = s0[uu].copy(), s1[uu].copy()
                    rz = zk - rinv * yk
                    zt = rz + rinv * sol
                    zr = alpha * zt + oma * zk
                    zn = zr + rinv * yk
                    zn = np.where(zn < pp0[uu], pp0[uu], zn)
                    zn = np.where(zn > pp1[uu], pp1[uu], zn)
                    yn = yk + rel_rho[k] * (zr - zn)
                    s0[uu], s1[uu] = zn, yn
                    X[i] = zn - rinv * yn
        else:
            for k in range(nrel):
                i = rel_i[k]
                uu = u0 + k
                X[i] = sigma * s0[uu] - pp0[uu] if rel_kind[k] == 0 else s0[uu] - rel_rinv[k] * s1[uu]
    # ---- stream_to_state_kernel + unscale
    x = np.zeros((lanes, plan.n), np.float32)
    z = np.zeros((lanes, plan.m), np.float32)
    y = np.zeros((lanes, plan.m), np.float32)
    for uu in range(n):
        o = sched["u_orig"][uu]
        if o < plan.n:
            x[:, o] = s0[uu]
        else:
            z[:, o - plan.n] = s0[uu]
            y[:, o - plan.n] = s1[uu]
    x = x * plan.scaling_d.astype(np.float32)
    z = z * plan.scaling_einv.astype(np.float32)
    y = y * plan.y_unscale.astype(np.float32)
    return x[:B], z[:B], y[:B]
