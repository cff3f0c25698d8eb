"""CPU replay of the TMA-fed per-call solve kernel (solve_stream.cu) over the
chunk tables the library builds (wmpc_solve_tables_host): every item's
copies and every work-vector index are checked against the kernel's buffer
sizes, and the replayed arithmetic (float32, the kernel's order) must equal
the oracle's serial solve bit for bit."""

import numpy as np
import pytest

from oracle import qdldl_ref
from warpmpc_b200 import problems, schedule

# the kernel's constants (solve_stream.cu)
BOX, CHUNK_ENTRIES, CHUNK_COLS, RHS_ROWS, TABLE_BYTES, STEP = 32, 64, 32, 96, 512, 8
DATA_ROWS = CHUNK_ENTRIES + CHUNK_COLS


def replay(qp, tab, lx, dinv, rhs):
    """One instance column at a time (lanes are independent); float32 throughout."""
    n, nnz_l = qp.n, qp.nnz_l
    T, D = tab["tables"], tab["desc"]
    f32 = np.float32
    # rows, the trash row (n: padded forward slots write it) and the zero row (n + 1)
    X = np.zeros(n + 2, dtype=f32)
    X[n] = np.nan  # never read by a real entry
    # rhs items: boxes of 32 rows inside the data area, rows past n zero-filled
    for k in range((n + RHS_ROWS - 1) // RHS_ROWS):
        r0 = k * RHS_ROWS
        rows = min(RHS_ROWS, n - r0)
        assert ((rows + BOX - 1) // BOX) * BOX <= DATA_ROWS
        for r in range(rows):
            X[qp.pinv[r0 + r]] = rhs[r0 + r]

    def chunk(k, backward):
        toff, words, e0, c0, E, C = (int(v) for v in D[k, :6])
        assert toff % 4 == 0 and words % 4 == 0 and words * 4 <= TABLE_BYTES
        assert 0 < C <= CHUNK_COLS and 0 <= E <= CHUNK_ENTRIES
        t = T[toff : toff + words]
        assert t[0] == C and t[1] == E and t[2] == c0 and t[3] == e0
        assert ((E + BOX - 1) // BOX) * BOX <= CHUNK_ENTRIES
        if backward:
            assert ((C + BOX - 1) // BOX) * BOX + CHUNK_ENTRIES <= DATA_ROWS
        cend = t[4 : 4 + C]
        roff = t[4 + C : 4 + C + E]
        assert np.all(roff % 128 == 0) and np.all(roff // 128 < n) and np.all(roff >= 0)
        assert np.all(np.diff(np.concatenate([[0], cend])) >= 0) and (C == 0 or cend[-1] == E)
        # a step reads up to STEP - 1 table words and L rows past the chunk's
        # last entry: still inside the table area and the stage's data rows
        assert (4 + C + E + STEP - 1) * 4 <= TABLE_BYTES and E + STEP - 1 <= DATA_ROWS
        L = np.full(DATA_ROWS, np.nan, dtype=f32)  # stale stage contents past the copied rows
        L[:E] = lx[e0 : e0 + E]  # rows past nnz_l would be zero-filled by the copy
        return c0, C, cend, roff // 128, L

    nch = D.shape[0]
    for k in range(nch):
        c0, C, cend, rows, L = chunk(k, False)
        b = 0
        with np.errstate(invalid="ignore"):
            for j in range(C):
                e = int(cend[j])
                if e > b:
                    val = X[c0 + j]
                    for q in range(b, e, STEP):
                        o = [int(rows[q + i]) if q + i < e else n for i in range(STEP)]
                        w = [X[o[i]] for i in range(STEP)]
                        for i in range(STEP):
                            X[o[i]] = f32(w[i] - f32(L[q + i] * val))
                b = e
    assert X[n + 1] == 0.0
    for k in range(nch - 1, -1, -1):
        c0, C, cend, rows, L = chunk(k, True)
        for j in range(C - 1, -1, -1):
            b = int(cend[j - 1]) if j > 0 else 0
            e = int(cend[j])
            corr = f32(0.0)
            for q in range(b, e, STEP):
                for i in range(STEP):
                    if q + i < e:
                        corr = f32(corr + f32(L[q + i] * X[rows[q + i]]))
                    else:  # L = 0 times the zero row
                        corr = f32(corr + f32(f32(0.0) * X[n + 1]))
            X[c0 + j] = f32(f32(X[c0 + j] * dinv[c0 + j]) - corr)
    # chunks cover every column exactly once, in order
    assert np.array_equal(np.concatenate([np.arange(d[3], d[3] + d[5]) for d in D]), np.arange(n))
    return X[qp.pinv]


@pytest.mark.parametrize("cls", [problems.SMALL, problems.CARTPOLE, problems.QUADROTOR], ids=lambda c: c.name)
def test_solve_stream_replay_matches_oracle(cls):
    from oracle import osqp_ref

    b = problems.make_batch(cls, 2, seed=21)
    plan = problems.make_plan(b)
    qp = plan.qdldl_plan
    tab = schedule.solve_tables(qp)
    kkt = osqp_ref.assemble_kkt_values(plan, b.p_values, b.a_values)  # (B, nnz_kkt) original order
    rng = np.random.default_rng(3)
    for i in range(2):
        lx, d, dinv = qdldl_ref.factor(qp, kkt[i : i + 1].T.astype(np.float32))
        rhs = rng.standard_normal((qp.n, 1)).astype(np.float32)
        want = qdldl_ref.solve(qp, lx, dinv, rhs)[:, 0]
        got = replay(qp, tab, lx[:, 0], dinv[:, 0], rhs[:, 0])
        np.testing.assert_array_equal(got, want)


def replay_factor(qp, sched, kkt):
    """The staged per-call factorization (factor_rows_kernel) for one
    instance: compact accumulator slots from the library's tables, L re-reads
    by position lp[c] + q, float32 in the kernel's order."""
    rg = sched["ragged"]
    pp, ip = np.asarray(rg["proc_ptr"]), np.asarray(rg["init_ptr"])
    pcols, poff, plidx = np.asarray(rg["proc_cols"]), np.asarray(rg["proc_offsets"]), np.asarray(rg["proc_lidx"])
    init_pos = np.asarray(rg["init_pos"])
    init_slot, upd_ptr, upd_slot = (np.asarray(sched[k]) for k in ("init_slot", "upd_ptr", "upd_slot"))
    n, f32 = qp.n, np.float32
    lx = np.full(qp.nnz_l, np.nan, dtype=f32)
    dinv = np.full(n, np.nan, dtype=f32)
    d = np.zeros(n, dtype=f32)
    for k in range(n):
        p0, p1, i0, i1 = pp[k], pp[k + 1], ip[k], ip[k + 1]
        ys = np.zeros(p1 - p0, dtype=f32)
        dk = f32(kkt[qp.perm_to_orig[qp.diag_pos[k]]])
        for e in range(i0, i1):
            s = init_slot[e]
            assert 0 <= s < p1 - p0
            ys[s] = f32(ys[s] + f32(kkt[qp.perm_to_orig[init_pos[e]]]))
        u = upd_ptr[p0]
        for e in range(p0, p1):
            c = pcols[e]
            val = ys[e - p0]
            for q in range(poff[e]):
                lid = qp.lp[c] + q
                assert lid < qp.lp[c + 1] and not np.isnan(lx[lid])  # written by an earlier row
                ys[upd_slot[u]] = f32(ys[upd_slot[u]] - f32(lx[lid] * val))
                u += 1
            assert not np.isnan(dinv[c])
            lval = f32(val * dinv[c])
            lx[plidx[e]] = lval
            dk = f32(dk - f32(val * lval))
        assert u == upd_ptr[p1]
        d[k] = dk
        dinv[k] = f32(f32(1.0) / dk)
    return lx, d, dinv


@pytest.mark.parametrize("cls", [problems.SMALL, problems.QUADROTOR], ids=lambda c: c.name)
def test_staged_factor_replay_matches_oracle(cls):
    from oracle import osqp_ref

    b = problems.make_batch(cls, 1, seed=23)
    plan = problems.make_plan(b)
    qp = plan.qdldl_plan
    sched = schedule.stream_schedule(plan)
    kkt = osqp_ref.assemble_kkt_values(plan, b.p_values, b.a_values)[0].astype(np.float32)
    lx, d, dinv = replay_factor(qp, sched, kkt)
    lx_o, d_o, dinv_o = qdldl_ref.factor(qp, kkt[:, None])
    np.testing.assert_array_equal(lx, lx_o[:, 0])
    np.testing.assert_array_equal(d, d_o[:, 0])
    np.testing.assert_array_equal(dinv, dinv_o[:, 0])
