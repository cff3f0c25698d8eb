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

KHDR = 8  # chunk meta header words
KUW = 8  # words per unit
FIRST, LAST, FWD = 1, 2, 4
DSHIFT = 8  # flags word: flags | D^-1 byte offset << 8
NSENT = 4  # sentinel units per chunk


def _f32(x):
    return np.float32(x)


def replay(plan, sched, p_values, a_values, q, l, u, x0=None, z0=None, y0=None, max_iter=None, lag=None):
    """Run the stream algorithm for a batch of <= 32 instances (float32).

    A frontier-slot schedule (``sched["frontier_slots"] > 0``) runs the form
    that schedule is built for: the work vector is a slot array, the
    right-hand sides live in a vector R read through each forward chunk's
    stage, the forward results (left by the forward units over their rows'
    right-hand sides in the stage, then copied out) in a vector Y read through
    each backward chunk's stage, and the releases of a backward chunk run ``lag`` chunks
    after it (the most a release may trail the sweep; default the schedule's
    lag) -- so a slot freed too early shows up as a wrong result."""
    qp = plan.qdldl_plan
    rg = sched["ragged"]
    n, nnz_l = qp.n, qp.nnz_l
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
    # ---- factor_stream_kernel (streams as flat float arrays; unit entries lane stride 4, D^-1 stride 1)
    lane = np.arange(lanes)
    BL, FL = sched["blen"], sched["flen"]
    Lb = np.full(BL, np.nan, dtype=np.float32)
    Fs = np.full(FL, np.nan, dtype=np.float32)

    def uidx(off, total):
        idx = off + 4 * lane
        assert off >= 0 and idx[-1] < total
        return idx

    def didx(off):
        idx = off + lane
        assert off >= 0 and idx[-1] < BL
        return idx

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
            base = sched["col_uoff"][c]
            u0 = sched["upd_ptr"][e]
            val = ys[e - p0].copy()
            for qq in range(off):
                s = sched["upd_slot"][u0 + qq]
                lv = Lb[uidx(base + (qq >> 2) * 128 + (qq & 3), BL)]
                assert 0 <= s < p1 - p0 and not np.isnan(lv).any()
                ys[s] = ys[s] - lv * val
            dv = Lb[didx(sched["dinv_off"][c])]
            assert not np.isnan(dv).any()
            lval = val * dv
            Lb[uidx(sched["proc_boff"][e], BL)] = lval
            fo = int(sched["proc_foff"][e])
            if fo >= 0:
                Fs[uidx(fo, FL)] = lval
            else:  # a releaser forward unit in the backward stream
                Lb[uidx(-1 - fo, BL)] = lval
            dk = dk - val * lval
        Lb[didx(sched["dinv_off"][k])] = _f32(1.0) / dk
    for off in sched["pad_boff"]:
        Lb[uidx(off, BL)] = 0.0
    for off in sched["pad_foff"]:
        Fs[uidx(off, FL)] = 0.0
    assert not np.isnan(Lb).any(), "backward stream positions not all written"
    assert not np.isnan(Fs).any(), "forward stream positions not all written"
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
    fr = int(sched.get("frontier_slots", 0)) > 0
    zr = int(sched["frontier_slots"]) if fr else n  # the zero row (slot); the trash row follows
    X = np.full((zr + 2, lanes), np.nan, dtype=np.float32)
    X[zr] = 0.0
    R = np.full((n, lanes), np.nan, dtype=np.float32)  # frontier: right-hand sides
    Y = np.full((n, lanes), np.nan, dtype=np.float32)  # frontier: forward results
    lag = (int(sched["frontier_lag"]) if fr else 1) if lag is None else lag
    meta_all = sched["meta"]
    fmeta_all = sched["fmeta"]
    nfc = sched["n_fchunks"]

    def block(all_, offs, words, ch, maxw):
        off, w = offs[ch], words[ch]
        assert w <= maxw and w % 4 == 0 and off % 4 == 0 and off + w <= all_.size
        return all_[off : off + w]

    def xrow(byte_off):
        assert byte_off % 128 == 0 and 0 <= byte_off // 128 <= zr + 1
        return byte_off // 128

    def run_units(m, nu, stage, backward, first_unit=0):
        """The consumer's unit loop: units are computed in groups of 3, unit
        u+1's operands loaded before unit u's arithmetic and store; units past
        nu are sentinels (zero-row reads, unit 0's L values, trash-row
        stores)."""
        ncomp = -(-nu // 3) * 3
        off = KHDR + first_unit * KUW
        assert 1 <= nu and off + (nu + NSENT) * KUW <= m.size and ncomp + 1 < nu + NSENT
        units = m[off : off + (nu + NSENT) * KUW].reshape(nu + NSENT, KUW)
        ubase = int(units[0][6]) // 512  # stage position of the list's first unit
        for sent in units[nu:]:
            assert np.all(sent[:4] == zr * 128) and sent[4] == (0 if fr else n * 128)
            assert sent[5] == 0 and sent[6] == 0 and sent[7] == (zr + 1) * 128
        nfl = stage.size

        def load(u):
            src, ctl = units[u, :4], units[u, 4:]
            lo = int(ctl[2])
            assert lo % 512 == 0 and lo // 4 + 128 <= nfl
            assert lo == ((ubase + u) * 512 if u < nu else 0)
            lv = stage[lo // 4 : lo // 4 + 128].reshape(lanes, 4).T.copy()  # [slot][lane]
            xs = [X[xrow(o)].copy() for o in src]
            if fr:  # t from the stage (right-hand-side block / forward-result block)
                to = int(ctl[0])
                assert to % 128 == 0 and to // 4 + 32 <= nfl
                t = stage[to // 4 : to // 4 + 32].copy()
            else:
                t = X[xrow(ctl[0])].copy()
            d = None
            if backward:
                doff = int(ctl[1]) >> DSHIFT
                assert doff % 4 == 0 and doff // 4 + 32 <= nfl
                d = stage[doff // 4 : doff // 4 + 32].copy()
            if u < nu and not fr:
                assert xrow(ctl[3]) == (xrow(ctl[0]) if int(ctl[1]) & LAST else n + 1)
            return ctl, lv, xs, t, d

        cur = load(0)
        acc = np.zeros(lanes, np.float32)
        prev = np.zeros(lanes, np.float32)
        with np.errstate(all="ignore"):
            for u in range(ncomp):
                nxt = load(u + 1)
                ctl, lv, xs, t, d = cur
                fl = int(ctl[1])
                if backward:
                    x0 = prev if fl & FWD else xs[0]
                    acc = np.zeros(lanes, np.float32) if fl & FIRST else acc
                    acc = acc + lv[0] * x0
                    acc = acc + lv[1] * xs[1]
                    acc = acc + lv[2] * xs[2]
                    acc = acc + lv[3] * xs[3]
                    res = t * d - acc
                else:
                    x3 = prev if fl & FWD else xs[3]
                    acc = t if fl & FIRST else acc
                    acc = acc - lv[0] * xs[0]
                    acc = acc - lv[1] * xs[1]
                    acc = acc - lv[2] * xs[2]
                    acc = acc - lv[3] * x3
                    res = acc
                X[xrow(ctl[3])] = res
                if fr and not backward:  # every unit also stores over its row's right-hand side in the stage
                    to = int(ctl[0])
                    stage[to // 4 : to // 4 + 32] = res
                prev = res
                cur = nxt

    pending = []  # deferred releases (frontier lag)
    items = [(0, nch - 1 - t) for t in range(nch)]
    for _ in range(iters):
        items += [(1, c) for c in range(nfc)] + [(2, c) for c in range(nch - 1, -1, -1)]
    for kind, ch in items:
        if kind == 1:
            fm = block(fmeta_all, sched["fmeta_off"], sched["fmeta_words"], ch, sched["max_fmeta_words"])
            nu = int(fm[0])
            assert nu == sched["fchunk_units"][ch] and nu <= sched["max_funits"]
            o0, o1 = sched["fchunk_off"][ch], sched["fchunk_off"][ch + 1]
            assert o1 - o0 == nu * 128 and o1 <= FL
            stage = Fs[o0:o1]
            if fr:  # the chunk's rows' right-hand sides follow its units
                r0, r1 = int(fm[1]), int(fm[2])
                assert 0 <= r0 < r1 <= n and r1 - r0 <= sched["max_frows"]
                assert not np.isnan(R[r0:r1]).any(), "a right-hand side is read before its release"
                stage = np.concatenate([stage, R[r0:r1].reshape(-1)])
            if fr:  # rows without entries: copied from the stage into their slots before the units
                ncopy = int(fm[3])
                c0 = KHDR + (nu + NSENT) * KUW
                assert c0 % 2 == 0 and c0 + 2 * ncopy <= fm.size
                for k in range(ncopy):
                    src, dst = int(fm[c0 + 2 * k]), int(fm[c0 + 2 * k + 1])
                    assert src % 128 == 0 and nu * 512 <= src and src // 4 + 32 <= stage.size
                    X[xrow(dst)] = stage[src // 4 : src // 4 + 32]
            if nu:
                run_units(fm, nu, stage, backward=False)
            if fr:  # the second releaser copies the block (now the rows' forward results) to Y
                Y[r0:r1] = stage[nu * 128 : nu * 128 + (r1 - r0) * 32].reshape(r1 - r0, lanes)
            continue
        m = block(meta_all, sched["meta_off"], sched["meta_words"], ch, sched["max_meta_words"])
        ns, ncols, nrel, c0, u0, nprim, nl, npre = (int(v) for v in m[:8])
        nu = ns + nl + npre
        assert nu == sched["chunk_units"][ch] and ncols == sched["chunk_cols"][ch] and nrel == sched["chunk_nrel"][ch]
        assert u0 == sched["chunk_u0"][ch] and nu <= sched["max_units"] and ncols <= sched["max_cols"]
        assert nrel <= sched["max_rel"] and 0 <= u0 and u0 + nrel <= n and 0 <= nprim <= nrel
        r = KHDR + (nu + 3 * NSENT) * KUW
        assert r + 4 * nrel <= m.size and r % 4 == 0
        recs = m[r : r + 4 * nrel].reshape(nrel, 4)
        rel_i = recs[:, 0].copy()
        rel_rho = recs[:, 1].copy().view(np.float32)
        rel_rinv = recs[:, 2].copy().view(np.float32)
        for k in range(nrel):
            assert (sched["u_orig"][u0 + k] < plan.n) == (k < nprim)
        o0, o1 = sched["chunk_off"][ch], sched["chunk_off"][ch + 1]
        assert o1 - o0 == nu * 128 + ncols * 32 and o1 <= BL
        stage = Lb[o0:o1]
        if fr:
            assert nl == 0 and npre == 0
            if kind == 2:  # the chunk's columns' forward results follow its D^-1 rows
                assert not np.isnan(Y[c0 : c0 + ncols]).any()
                stage = np.concatenate([stage, Y[c0 : c0 + ncols].reshape(-1)])
        leaf_at, pre_at = ns + NSENT, ns + nl + 2 * NSENT
        if kind == 0:
            # the first-right-hand-side pass copies only the releaser's forward units
            assert sched["chunk_pre_u0"][ch] == ns + nl and sched["chunk_pre_units"][ch] == npre
            stage = np.full_like(stage, np.nan)
            p0, p1 = (ns + nl) * 128, (ns + nl + npre) * 128
            stage[p0:p1] = Lb[o0 + p0 : o0 + p1]
        def rhs_out(k, i, value):
            """The next right-hand side: into R (frontier) or the work vector."""
            if fr:
                idx = int(recs[k, 3])
                assert 0 <= idx < n
                R[idx] = value
            else:
                X[i] = value

        def releases(recs=recs, rel_i=rel_i, rel_rho=rel_rho, rel_rinv=rel_rinv, u0=u0, nprim=nprim, nrel=nrel):
            for k in range(nrel):
                i = xrow(rel_i[k])
                assert i < (zr if fr else n)
                uu = u0 + k
                sol = X[i].copy()
                assert not np.isnan(sol).any()
                if k < nprim:
                    xn = alpha * sol + oma * s0[uu]
                    s0[uu] = xn
                    out = sigma * xn - pp0[uu]
                else:
                    rinv = rel_rinv[k]
                    zk, yk = s0[uu].copy(), s1[uu].copy()
                    rz = zk - rinv * yk
                    zt = rz + rinv * sol
                    zrel = alpha * zt + oma * zk
                    zn = zrel + rinv * yk
                    zn = np.where(zn < pp0[uu], pp0[uu], zn)
                    zn = np.where(zn > pp1[uu], pp1[uu], zn)
                    yn = yk + rel_rho[k] * (zrel - zn)
                    s0[uu], s1[uu] = zn, yn
                    out = zn - rinv * yn
                if fr:
                    R[int(recs[k, 3])] = out
                else:
                    X[i] = out

        if kind == 2:
            if ns:
                run_units(m, ns, stage, backward=True)
            if nl:
                run_units(m, nl, stage, backward=True, first_unit=leaf_at)
            pending.append(releases)
            # a release may trail the sweep by lag - 1 chunks; all are done before the forward sweep
            while len(pending) > max(lag - 1, 0) or (ch == 0 and pending):
                pending.pop(0)()
        else:
            for k in range(nrel):
                i = -1 if fr else xrow(rel_i[k])
                uu = u0 + k
                rhs_out(k, i, sigma * s0[uu] - pp0[uu] if k < nprim else s0[uu] - rel_rinv[k] * s1[uu])
        if npre:
            run_units(m, npre, stage, backward=False, first_unit=pre_at)
        assert X[zr].max() == 0.0 and X[zr].min() == 0.0
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
