"""ctypes binding of the oracle's C restatement (oracle/c/osqp_cpu.c).

TEST INFRASTRUCTURE ONLY (oracle): the CPU baseline that bench.py times and a
cross-check of the NumPy oracle.  Built with ``make -C oracle``.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "libosqp_cpu.so"
LIB64 = HERE / "_build" / "libosqp_cpu_f64.so"

_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)


_rp = _f32p  # rebound per precision below


class _Pattern(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("nnz_a", ctypes.c_int), ("nnz_l", ctypes.c_int)] + [
        (k, _i32p)
        for k in ("perm_to_orig", "diag_pos", "init_ptr", "init_rows", "init_pos", "proc_ptr", "proc_cols",
                  "proc_lidx", "proc_offsets", "lp", "li", "p", "pinv")
    ]


def _osqp_struct(real, rp):
    class _Osqp(ctypes.Structure):
        _fields_ = [
            ("n", ctypes.c_int), ("m", ctypes.c_int), ("nnz_p", ctypes.c_int), ("nnz_a", ctypes.c_int),
            ("nnz_kkt", ctypes.c_int), ("nnz_pf", ctypes.c_int), ("sigma", real), ("alpha", real),
            ("kkt_base", rp), ("kkt_src", _i32p), ("p_scale", rp), ("p_diag_sigma", rp), ("a_scale", rp),
            ("a_row_ptr", _i32p), ("a_row_ent", _i32p), ("a_rows", _i32p), ("a_cols", _i32p), ("a_col_ptr", _i32p),
            ("pf_row_ptr", _i32p), ("pf_val", _i32p), ("pf_col", _i32p),
            ("rho", rp), ("rho_inv", rp), ("q_scale", rp), ("scaling_d", rp), ("scaling_dinv", rp),
            ("scaling_e", rp), ("scaling_einv", rp), ("y_scale", rp), ("y_unscale", rp),
        ]

    return _Osqp


_f64p = ctypes.POINTER(ctypes.c_double)
_Osqp32 = _osqp_struct(ctypes.c_float, _f32p)
_Osqp64 = _osqp_struct(ctypes.c_double, _f64p)


def build(force: bool = False) -> pathlib.Path:
    src = HERE / "c" / "osqp_cpu.c"
    stale = lambda p: not p.exists() or p.stat().st_mtime < src.stat().st_mtime  # noqa: E731
    if force or stale(LIB) or stale(LIB64):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


class CpuOSQP:
    """The C restatement bound to one FixedOSQPPlan."""

    def __init__(self, plan, dtype=np.float32):
        build()
        self.dtype = np.dtype(dtype)
        double = self.dtype == np.float64
        self.lib = ctypes.CDLL(str(LIB64 if double else LIB))
        self._fn = self.lib.oc_osqp_solve_f64 if double else self.lib.oc_osqp_solve
        self._fn.restype = ctypes.c_int
        self._rp = _f64p if double else _f32p
        self.plan = plan
        from warpmpc_b200.jax_qdldl.planning import plan_ragged_program

        qp = plan.qdldl_plan
        rg = plan_ragged_program(qp)
        keep = self._keep = []

        def i(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
            keep.append(a)
            return a.ctypes.data_as(_i32p)

        def f(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=self.dtype))
            keep.append(a)
            return a.ctypes.data_as(self._rp)

        self.pat = _Pattern(qp.n, qp.nnz_a, qp.nnz_l, i(qp.perm_to_orig), i(qp.diag_pos), i(rg["init_ptr"]),
                            i(rg["init_rows"]), i(rg["init_pos"]), i(rg["proc_ptr"]), i(rg["proc_cols"]),
                            i(rg["proc_lidx"]), i(rg["proc_offsets"]), i(qp.lp), i(qp.li), i(qp.p), i(qp.pinv))
        n, m = plan.n, plan.m
        kkt_src = np.full(plan.nnz_kkt, -1, dtype=np.int32)
        kkt_src[plan.p_to_kkt] = np.arange(plan.nnz_p)
        kkt_src[plan.a_to_kkt] = plan.nnz_p + np.arange(plan.nnz_a)
        a_row_ent = np.argsort(plan.a_rows, kind="stable").astype(np.int32)
        a_row_ptr = np.concatenate([[0], np.cumsum(np.bincount(plan.a_rows, minlength=m))]).astype(np.int32)
        a_col_ptr = np.concatenate([[0], np.cumsum(np.bincount(plan.a_cols, minlength=n))]).astype(np.int32)
        pf_order = np.argsort(plan.p_full_rows, kind="stable")
        pf_row_ptr = np.concatenate([[0], np.cumsum(np.bincount(plan.p_full_rows, minlength=n))]).astype(np.int32)
        s = plan.settings
        osqp_cls = _Osqp64 if double else _Osqp32
        self.osqp = osqp_cls(
            n, m, plan.nnz_p, plan.nnz_a, plan.nnz_kkt, int(plan.p_full_rows.size), self.dtype.type(s.sigma),
            self.dtype.type(s.alpha), f(plan.kkt_upper.data), i(kkt_src), f(plan.p_scale), f(plan.p_diag_sigma),
            f(plan.a_scale), i(a_row_ptr), i(a_row_ent), i(plan.a_rows), i(plan.a_cols), i(a_col_ptr),
            i(pf_row_ptr), i(plan.p_full_value_map[pf_order]), i(plan.p_full_cols[pf_order]),
            f(plan.rho_vec), f(plan.rho_inv_vec), f(plan.q_scale), f(plan.scaling_d), f(plan.scaling_dinv),
            f(plan.scaling_e), f(plan.scaling_einv), f(plan.y_scale), f(plan.y_unscale),
        )

    def solve(self, p_values, a_values, q, l, u, warm=None, max_iter=None, threads: int | None = None):
        plan = self.plan
        c = lambda a: np.ascontiguousarray(np.asarray(a, dtype=self.dtype))  # noqa: E731
        p_values, a_values, q, l, u = (np.atleast_2d(c(v)) for v in (p_values, a_values, q, l, u))
        batch = q.shape[0]
        dt = self.dtype
        x = np.empty((batch, plan.n), dt)
        z = np.empty((batch, plan.m), dt)
        y = np.empty((batch, plan.m), dt)
        prim = np.empty(batch, dt)
        dual = np.empty(batch, dt)
        obj = np.empty(batch, dt)
        fp = lambda a: None if a is None else a.ctypes.data_as(self._rp)  # noqa: E731
        w = [None, None, None] if warm is None else [c(v) for v in warm]
        threads = threads or os.cpu_count() or 1
        iters = int(plan.settings.max_iter if max_iter is None else max_iter)

        def run(lo, hi):
            # ctypes releases the GIL for the duration of the call
            return self._fn(
                ctypes.byref(self.pat), ctypes.byref(self.osqp), lo, hi, iters,
                fp(p_values), p_values.shape[0], fp(a_values), a_values.shape[0], fp(q), fp(l), fp(u),
                fp(w[0]), fp(w[1]), fp(w[2]), fp(x), fp(z), fp(y), fp(prim), fp(dual), fp(obj),
            )

        chunks = np.linspace(0, batch, min(threads, max(batch, 1)) + 1).astype(int)
        with ThreadPoolExecutor(max_workers=threads) as pool:
            codes = list(pool.map(lambda ab: run(int(ab[0]), int(ab[1])), zip(chunks[:-1], chunks[1:])))
        if any(codes):
            raise RuntimeError("oc_osqp_solve failed")
        self.threads_used = len(codes)
        return x, z, y, prim, dual, obj
