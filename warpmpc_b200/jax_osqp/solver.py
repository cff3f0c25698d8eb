"""Compiled batched OSQP-ADMM on the CUDA library.

Mirror of ``compile_osqp`` (``warpmpc/jax_osqp/solver.py:685-1492``) with
``qdldl_backend="cuda"``.  All callables take and return ``torch`` tensors
(batch-major ``(B, .)`` like the reference; P/A value batches of one are
broadcast).  Two execution modes share one C-ABI call:

* ``mode="persistent"`` (default): one fused launch per instance tile --
  KKT assembly, factorization, all ``max_iter`` ADMM iterations (optionally
  with OSQP's termination test every ``check_termination`` iterations) and
  the residual epilogue;
* ``mode="plain"``: the reference's loop structure with the CUDA factor and
  solve as drop-in kernels (one factor, then per iteration one solve launch
  and one ADMM-update launch), i.e. what ``qdldl_backend="cuda"`` gives the
  unchanged reference ADMM loop.

Arithmetic is float32 in the reference's operation order.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import native
from ..jax_qdldl.core import DevicePlan, _as_f32, _workspace, compile_qdldl_variant
from .types import CompiledOSQP, FixedOSQPPlan, OSQPWarmStart


def values_for_compiled_qdldl(compiled, kkt_values):
    """(B, nnz) -> the compiled QDLDL's values layout (solver.py:665-670)."""
    if compiled.values_layout == "original_batch":
        return kkt_values
    if compiled.values_layout == "original_symbolic":
        return kkt_values.T
    raise ValueError(f"unknown QDLDL values layout {compiled.values_layout}")


def rhs_for_compiled_qdldl(compiled, rhs):
    """(B, n) -> the compiled QDLDL's rhs layout (solver.py:673-678)."""
    if compiled.rhs_layout == "batch":
        return rhs
    if compiled.rhs_layout == "symbolic":
        return rhs.T
    raise ValueError(f"unknown QDLDL rhs layout {compiled.rhs_layout}")


def batch_from_compiled_qdldl(compiled, values):
    return values.T if compiled.rhs_layout == "symbolic" else values


class DeviceOSQP:
    """A FixedOSQPPlan uploaded to one device (``wmpc_osqp``) plus its KKT plan."""

    def __init__(self, plan: FixedOSQPPlan, device=None, kkt_plan: DevicePlan | None = None):
        self.plan = plan
        self.kkt = kkt_plan if kkt_plan is not None else DevicePlan(plan.qdldl_plan, device)
        self.device_index = self.kkt.device_index
        s = plan.settings
        keep = {
            "kkt_base": native.f32(plan.kkt_upper.data),
            "p_to_kkt": native.i32(plan.p_to_kkt),
            "p_diag_sigma": native.f32(plan.p_diag_sigma),
            "a_to_kkt": native.i32(plan.a_to_kkt),
            "p_scale": native.f32(plan.p_scale),
            "a_scale": native.f32(plan.a_scale),
            "a_rows": native.i32(plan.a_rows),
            "a_cols": native.i32(plan.a_cols),
            "p_full_rows": native.i32(plan.p_full_rows),
            "p_full_cols": native.i32(plan.p_full_cols),
            "p_full_value_map": native.i32(plan.p_full_value_map),
            "rho_vec": native.f32(plan.rho_vec),
            "rho_inv_vec": native.f32(plan.rho_inv_vec),
            "q_scale": native.f32(plan.q_scale),
            "scaling_d": native.f32(plan.scaling_d),
            "scaling_dinv": native.f32(plan.scaling_dinv),
            "scaling_e": native.f32(plan.scaling_e),
            "scaling_einv": native.f32(plan.scaling_einv),
            "y_scale": native.f32(plan.y_scale),
            "y_unscale": native.f32(plan.y_unscale),
            "rho_type": native.i32(plan.constr_type),
            "rho_to_kkt": native.i32(plan.rho_to_kkt),
        }
        kw = {}
        for k, v in keep.items():
            kw[k] = native.ptr_f32(v) if v.dtype == np.float32 else native.ptr_i32(v)
        desc = native.OsqpDesc(
            n=plan.n, m=plan.m, nnz_p=plan.nnz_p, nnz_a=plan.nnz_a, nnz_kkt=plan.nnz_kkt,
            sigma=np.float32(s.sigma), alpha=np.float32(s.alpha), rho=np.float32(s.rho),
            nnz_p_full=int(plan.p_full_rows.size), **kw,
        )
        handle = ctypes.c_void_p()
        native.check(native.lib().wmpc_osqp_create(ctypes.byref(desc), self.kkt.handle, ctypes.byref(handle)))
        self.handle = handle

    @property
    def torch_device(self):
        return self.kkt.torch_device

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                native.lib().wmpc_osqp_destroy(handle)
            except Exception:  # pragma: no cover
                pass
            self.handle = None


_MODES = {"plain": native.WMPC_OSQP_PLAIN, "persistent": native.WMPC_OSQP_PERSISTENT}


class OSQPEngine:
    """Host-side driver of ``wmpc_osqp_factor`` / ``wmpc_osqp_solve``.

    A plan with ``settings.adaptive_rho`` runs either the per-call ("plain")
    kernels or, in "persistent" mode where the pattern has the streaming
    schedule, the streaming kernels in launches of ``adaptive_rho_interval``
    iterations with a per-instance rho (the same iterates, rho and refactor
    counts); other modes fall back to "plain".  Rho adaptation runs fixed
    iterations on the persistent path (``check_termination`` 0)."""

    def __init__(self, plan: FixedOSQPPlan, device=None, mode: str = "persistent", kkt_plan: DevicePlan | None = None):
        if mode not in _MODES:
            raise ValueError(f"unknown mode {mode!r}; expected one of {sorted(_MODES)}")
        self.plan = plan
        self.dev = DeviceOSQP(plan, device, kkt_plan=kkt_plan)
        self.mode = mode
        if plan.settings.adaptive_rho and not (mode == "persistent" and self.stream_info()["streaming"]
                                               and not plan.settings.check_termination):
            self.mode = "plain"
        self.device = self.dev.torch_device
        self.last_iters = None
        self.last_status = None
        self.last_rho = None
        self.last_rho_updates = None

    def workspace_bytes(self, batch: int, keep_factor: bool = False) -> int:
        """Device workspace bytes of a solve of ``batch`` instances (factoring;
        ``keep_factor``: enough for the adjoint on the kept factorization)."""
        lib = native.lib()
        mode_id = _MODES[self.mode]
        if keep_factor:
            return int(lib.wmpc_osqp_adjoint_workspace_bytes(self.dev.handle, batch, mode_id))
        return int(lib.wmpc_osqp_workspace_bytes(self.dev.handle, batch, mode_id, 0))

    def stream_info(self) -> dict:
        """The streaming schedule this problem carries: ``streaming`` (persistent
        solves run the streaming kernel), ``frontier_slots`` (work-vector slots
        of the frontier form; 0 for the plain form), ``n`` (KKT dimension) and
        ``frontier_lag``."""
        info = (ctypes.c_int32 * 4)()
        native.check(native.lib().wmpc_osqp_stream_info(self.dev.handle, info))
        return {"streaming": bool(info[0]), "frontier_slots": int(info[1]), "n": int(info[2]),
                "frontier_lag": int(info[3])}

    # -- argument normalisation -------------------------------------------------
    def _mat(self, values, width, name):
        t = _as_f32(values, self.device, name)
        if t.dim() == 1:
            t = t[None, :]
        if t.dim() != 2 or t.shape[1] != width:
            raise ValueError(f"{name} must have shape (batch, {width}) or ({width},)")
        return t.contiguous()

    def _vec(self, values, width, batch, name):
        t = self._mat(values, width, name)
        if t.shape[0] == 1 and batch > 1:
            t = t.expand(batch, width).contiguous()
        if t.shape[0] != batch:
            raise ValueError(f"{name} has batch {t.shape[0]}, expected {batch}")
        return t

    def factor(self, p_values, a_values):
        import torch

        pl = self.plan
        p = self._mat(p_values, pl.nnz_p, "p_values")
        a = self._mat(a_values, pl.nnz_a, "a_values")
        pb, ab = int(p.shape[0]), int(a.shape[0])
        if pb != 1 and ab != 1 and pb != ab:
            raise ValueError("p_values and a_values batches must match (or be 1)")
        fb = max(pb, ab)
        nk = pl.qdldl_plan.n
        lx = torch.empty((pl.qdldl_plan.nnz_l, fb), dtype=torch.float32, device=self.device)
        d = torch.empty((nk, fb), dtype=torch.float32, device=self.device)
        dinv = torch.empty((nk, fb), dtype=torch.float32, device=self.device)
        lib = native.lib()
        ws, wsb = _workspace(lib.wmpc_osqp_workspace_bytes(self.dev.handle, fb, _MODES[self.mode], 0), self.device)
        native.check(lib.wmpc_osqp_factor(self.dev.handle, p.data_ptr(), pb, a.data_ptr(), ab, lx.data_ptr(),
                                          d.data_ptr(), dinv.data_ptr(), native.tensor_ptr(ws), wsb,
                                          native.current_stream_handle(self.device)))
        return lx, dinv

    def _batch_args(self, p_values, a_values, q, l, u, warm, max_iter, check_termination, out):
        """The C batch descriptor, options, tensors to keep alive and outputs of one solve."""
        import torch

        pl = self.plan
        s = pl.settings
        p = self._mat(p_values, pl.nnz_p, "p_values")
        a = self._mat(a_values, pl.nnz_a, "a_values")
        qm = self._mat(q, pl.n, "q")
        batch = max(int(qm.shape[0]), int(p.shape[0]), int(a.shape[0]))
        for t, name in ((p, "p_values"), (a, "a_values")):
            if t.shape[0] not in (1, batch):
                raise ValueError(f"{name} batch must be 1 or {batch}")
        qm = self._vec(qm, pl.n, batch, "q")
        lm = self._vec(l, pl.m, batch, "l")
        um = self._vec(u, pl.m, batch, "u")
        dev = self.device
        if out is None:
            x = torch.empty((batch, pl.n), dtype=torch.float32, device=dev)
            z = torch.empty((batch, pl.m), dtype=torch.float32, device=dev)
            y = torch.empty((batch, pl.m), dtype=torch.float32, device=dev)
            prim = torch.empty(batch, dtype=torch.float32, device=dev)
            dual = torch.empty(batch, dtype=torch.float32, device=dev)
            obj = torch.empty(batch, dtype=torch.float32, device=dev)
            iters = torch.empty(batch, dtype=torch.int32, device=dev)
            status = torch.empty(batch, dtype=torch.int32, device=dev)
        else:
            x, z, y, prim, dual, obj, iters, status = out
            shapes = [(batch, pl.n), (batch, pl.m), (batch, pl.m), (batch,), (batch,), (batch,), (batch,), (batch,)]
            for t, shp in zip(out, shapes):
                if tuple(t.shape) != shp or not t.is_contiguous() or t.device != dev:
                    raise ValueError("out tensors have the wrong shape, layout or device")
        keep = [p, a, qm, lm, um]
        if warm is not None:
            wx = self._vec(warm[0], pl.n, batch, "warm_start_x")
            wz = self._vec(warm[1], pl.m, batch, "warm_start_z")
            wy = self._vec(warm[2], pl.m, batch, "warm_start_y")
            keep += [wx, wz, wy]
            x0, z0, y0 = wx.data_ptr(), wz.data_ptr(), wy.data_ptr()
        else:
            x0 = z0 = y0 = None
        data = native.OsqpBatch(
            batch=batch, p_values=p.data_ptr(), p_batch=int(p.shape[0]), a_values=a.data_ptr(),
            a_batch=int(a.shape[0]), q=qm.data_ptr(), l=lm.data_ptr(), u=um.data_ptr(), x0=x0, z0=z0, y0=y0,
            x=x.data_ptr(), z=z.data_ptr(), y=y.data_ptr(), prim_res=prim.data_ptr(), dual_res=dual.data_ptr(),
            obj=obj.data_ptr(), iters=iters.data_ptr(), status=status.data_ptr(),
        )
        opts = native.OsqpOptions(
            max_iter=int(s.max_iter if max_iter is None else max_iter),
            check_termination=int(s.check_termination if check_termination is None else check_termination),
            eps_abs=np.float32(s.eps_abs), eps_rel=np.float32(s.eps_rel), warm_start=1 if warm is not None else 0,
            adaptive_rho_interval=int(s.adaptive_rho_interval) if s.adaptive_rho else 0,
            adaptive_rho_tolerance=np.float32(s.adaptive_rho_tolerance),
        )
        return data, opts, keep, (x, z, y, prim, dual, obj, iters, status), batch

    def solve(self, p_values, a_values, q, l, u, warm=None, factor=None, max_iter=None, check_termination=None,
              mode=None, out=None, keep_factor=False, workspace=None):
        """Batched solve; returns ``(x, z, y, prim_res, dual_res, obj_val)``.

        ``out`` optionally supplies those six output tensors (plus ``iters``,
        ``status`` int32) to write into; warm-start inputs may alias ``out``
        (they are consumed before the outputs are written), which lets a CUDA
        graph chain solves without copies.  ``workspace`` optionally supplies
        the device workspace (a uint8 tensor of at least ``workspace_bytes``,
        or ``adjoint_workspace_bytes`` with ``keep_factor``) instead of a new
        allocation per call: a caller that chains solves (an SQP loop, a CUDA
        graph) keeps one; a kept factorization lives in it until the next
        solve that is given the same workspace.
        """
        pl = self.plan
        dev = self.device
        data, opts, keep, outs, batch = self._batch_args(p_values, a_values, q, l, u, warm, max_iter,
                                                         check_termination, out)
        x, z, y, prim, dual, obj, iters, status = outs
        mode_id = _MODES[self.mode if mode is None else mode]
        lib = native.lib()
        if factor is not None:
            lx, dinv = factor
            lx = _as_f32(lx, dev, "lx")
            dinv = _as_f32(dinv, dev, "dinv")
            fb = int(lx.shape[1])
            if lx.shape[0] != pl.qdldl_plan.nnz_l or dinv.shape != (pl.qdldl_plan.n, fb) or fb not in (1, batch):
                raise ValueError("lx/dinv do not match the plan or the batch")
            lx_p, dinv_p, ext = lx.data_ptr(), dinv.data_ptr(), 1
            keep += [lx, dinv]
        else:
            lx_p = dinv_p = None
            fb, ext = 0, 0
        if keep_factor:
            if factor is not None:
                raise ValueError("keep_factor needs the solve to factor (no external factor)")
            need = lib.wmpc_osqp_adjoint_workspace_bytes(self.dev.handle, batch, mode_id)
        else:
            need = lib.wmpc_osqp_workspace_bytes(self.dev.handle, batch, mode_id, ext)
        if workspace is not None:
            if workspace.device != dev or workspace.numel() * workspace.element_size() < need:
                raise ValueError(f"workspace must be a device tensor of at least {need} bytes on {dev}")
            ws, wsb = workspace, int(workspace.numel() * workspace.element_size())
        else:
            ws, wsb = _workspace(need, dev)
        if pl.settings.adaptive_rho:
            # each instance's final rho and number of rho changes (refactorizations)
            import torch

            rho_out = torch.empty(batch, dtype=torch.float32, device=dev)
            upd_out = torch.empty(batch, dtype=torch.int32, device=dev)
            data.rho, data.rho_updates = rho_out.data_ptr(), upd_out.data_ptr()
            self.last_rho, self.last_rho_updates = rho_out, upd_out
        native.check(lib.wmpc_osqp_solve(self.dev.handle, ctypes.byref(opts), ctypes.byref(data), lx_p, dinv_p, fb,
                                         mode_id, native.tensor_ptr(ws), wsb, native.current_stream_handle(dev)))
        self.last_iters = iters
        self.last_status = status
        self.last_workspace = (ws, wsb, mode_id, int(opts.check_termination)) if keep_factor else None
        return x, z, y, prim, dual, obj

    def solve_host(self, p_values, a_values, q, l, u, warm=None, out=None, chunks=4, max_iter=None,
                   check_termination=None, granule=None, first_fraction=0.15, on_slice=None):
        """Batched solve of host (CPU) tensors into host tensors, transfers overlapped with the solves.

        The batch is cut into ``chunks`` slices with boundaries on whole waves
        of 32-instance tiles over the device's SMs (``granule`` overrides that
        unit of 32 x the SM count); slice k's host-to-device copy runs on a
        copy stream while slice k-1 is solved on the current stream, and slice
        k-1's results go back on a second copy stream while slice k is
        solved.  Each slice pays the factorization's latency floor once, so
        few slices; ``first_fraction`` sizes the first slice, whose copy in
        nothing hides; the rest are equal (None: all equal).  Measured on the
        quadrotor workload (65,536 instances, closed loop, host advance
        included) with earlier, slower kernels: 4 slices with a 0.15 first
        slice 109 ms per step, 3 with 0.15 113 ms, 2 with 0.3 127 ms, one 142
        ms; with the current kernels the default takes 94.5 ms per step (the
        host advance in ``on_slice``).  Each slice is an ordinary ``solve`` of its instances, so
        the results equal a one-shot ``solve`` of the whole batch bit for bit.
        Inputs should be in pinned memory (pageable tensors still work, without
        the overlap).  ``out`` optionally gives the six host output tensors
        ``(x, z, y, prim_res, dual_res, obj_val)``; otherwise they are
        allocated pinned; the warm start may alias them (each slice's start is
        copied in before its results are copied out).  Returns them once the
        results are on the host (the
        call synchronizes the current stream); ``last_iters`` and
        ``last_status`` are host tensors afterwards.  ``on_slice(s0, s1)``, if
        given, is called for each slice in order as soon as its results are on
        the host, while the later slices are still being solved (a closed loop
        can advance those instances meanwhile); it may rewrite the host input
        rows [s0, s1), whose copies are done, and no other rows.
        """
        import torch

        pl = self.plan
        dev = self.device

        def host(t, width, name):
            if not isinstance(t, torch.Tensor):
                t = torch.as_tensor(np.asarray(t, dtype=np.float32))
            if t.device.type != "cpu" or t.dtype != torch.float32:
                raise ValueError(f"{name} must be a float32 host tensor")
            t = t if t.dim() == 2 else t.reshape(1, -1)
            if t.shape[1] != width:
                raise ValueError(f"{name} must have shape (batch, {width}) or ({width},)")
            return t.contiguous()

        p = host(p_values, pl.nnz_p, "p_values")
        a = host(a_values, pl.nnz_a, "a_values")
        qh, lh, uh = host(q, pl.n, "q"), host(l, pl.m, "l"), host(u, pl.m, "u")
        wh = None if warm is None else (host(warm[0], pl.n, "warm_start_x"), host(warm[1], pl.m, "warm_start_z"),
                                        host(warm[2], pl.m, "warm_start_y"))
        rows = [p, a, qh, lh, uh] + ([] if wh is None else list(wh))
        batch = max(int(t.shape[0]) for t in rows)
        for t, name in zip(rows, ("p_values", "a_values", "q", "l", "u", "warm_start_x", "warm_start_z",
                                  "warm_start_y")):
            if t.shape[0] not in (1, batch):
                raise ValueError(f"{name} batch must be 1 or {batch}")
        shapes = [(batch, pl.n), (batch, pl.m), (batch, pl.m), (batch,), (batch,), (batch,)]
        if out is None:
            out = tuple(torch.empty(s, dtype=torch.float32).pin_memory() for s in shapes)
        else:
            out = tuple(out)
            if len(out) != 6 or any(tuple(t.shape) != s or t.device.type != "cpu" or not t.is_contiguous()
                                    or t.dtype != torch.float32 for t, s in zip(out, shapes)):
                raise ValueError("out must be six contiguous float32 host tensors (x, z, y, prim, dual, obj)")
        iters_h = torch.empty(batch, dtype=torch.int32).pin_memory()
        status_h = torch.empty(batch, dtype=torch.int32).pin_memory()
        if batch == 0:
            return out
        # slice boundaries on whole waves of tiles (a partial wave costs a whole one)
        wave = int(granule) if granule else 32 * torch.cuda.get_device_properties(dev).multi_processor_count
        waves = -(-batch // wave)
        k = max(1, min(int(chunks), waves))
        if first_fraction is not None and k > 1:
            w1 = min(waves - (k - 1), max(1, int(round(waves * float(first_fraction)))))
            bounds = [0] + [min(batch, wave * (w1 + (waves - w1) * i // (k - 1))) for i in range(k)]
        else:
            bounds = [min(batch, wave * (waves * i // k)) for i in range(k + 1)]
        bounds[-1] = batch
        size = max(bounds[i + 1] - bounds[i] for i in range(k))

        cur = torch.cuda.current_stream(dev)
        if getattr(self, "_copy_streams", None) is None:
            self._copy_streams = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
        up, down = self._copy_streams
        start = torch.cuda.Event()
        start.record(cur)
        up.wait_event(start)
        down.wait_event(start)

        def dbuf(t, rows_):
            return torch.empty((rows_ if t.shape[0] == batch else 1, t.shape[1]), dtype=torch.float32, device=dev)

        sets = []
        for _ in range(min(2, k)):
            ins = [dbuf(t, size) for t in rows]
            outs = [torch.empty((size,) + s[1:], dtype=torch.float32, device=dev) for s in shapes]
            outs += [torch.empty(size, dtype=torch.int32, device=dev) for _ in range(2)]
            sets.append((ins, outs))
        in_ready, solved, copied = [], [], []
        for i in range(k):
            s0, s1 = bounds[i], bounds[i + 1]
            n = s1 - s0
            ins, outs = sets[i % 2]
            if i >= 2:
                up.wait_event(solved[i - 2])  # the set's inputs were read by slice i - 2
            with torch.cuda.stream(up):
                for h, d in zip(rows, ins):
                    if h.shape[0] == batch:
                        d[:n].copy_(h[s0:s1], non_blocking=True)
                    elif i < 2:
                        d.copy_(h, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(up)
            in_ready.append(ev)
            cur.wait_event(ev)
            if i >= 2:
                cur.wait_event(copied[i - 2])  # the set's outputs went back for slice i - 2
            dv = [d if d.shape[0] == 1 else d[:n] for d in ins]
            o = tuple(t[:n] for t in outs)
            self.solve(dv[0], dv[1], dv[2], dv[3], dv[4], warm=None if wh is None else tuple(dv[5:8]),
                       max_iter=max_iter, check_termination=check_termination, out=o)
            ev = torch.cuda.Event()
            ev.record(cur)
            solved.append(ev)
            down.wait_event(ev)
            with torch.cuda.stream(down):
                for h, d in zip(list(out) + [iters_h, status_h], o):
                    h[s0:s1].copy_(d, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(down)
            copied.append(ev)
        if on_slice is not None:
            for i in range(k):
                copied[i].synchronize()
                on_slice(bounds[i], bounds[i + 1])
        cur.wait_event(copied[-1])
        cur.wait_event(in_ready[-1])
        cur.synchronize()
        self.last_iters = iters_h
        self.last_status = status_h
        return out

    def adjoint(self, workspace, p_values, a_values, l, u, x, z, y, dx, dy=None, max_iter=None, residual=False):
        """Reverse-mode derivatives on the factor kept by ``solve(keep_factor=True)``.

        Returns ``(dq, dl, du, dp, da)`` per instance (``dp``/``da`` batch-major
        on P's upper pattern and A's pattern).  ``residual=True`` also forms
        the differential QP's primal residual (``last_adjoint_residual``),
        which costs a pass over P and A.
        """
        import torch

        ws, wsb, mode_id, check = workspace
        pl = self.plan
        p = self._mat(p_values, pl.nnz_p, "p_values")
        a = self._mat(a_values, pl.nnz_a, "a_values")
        x = self._mat(x, pl.n, "x")
        batch = int(x.shape[0])
        z = self._vec(z, pl.m, batch, "z")
        y = self._vec(y, pl.m, batch, "y")
        lm = self._vec(l, pl.m, batch, "l")
        um = self._vec(u, pl.m, batch, "u")
        dxm = self._vec(dx, pl.n, batch, "dx")
        dym = None if dy is None else self._vec(dy, pl.m, batch, "dy")
        dev = self.device
        dq = torch.empty((batch, pl.n), dtype=torch.float32, device=dev)
        dl = torch.empty((batch, pl.m), dtype=torch.float32, device=dev)
        du = torch.empty((batch, pl.m), dtype=torch.float32, device=dev)
        dp = torch.empty((batch, pl.nnz_p), dtype=torch.float32, device=dev)
        da = torch.empty((batch, pl.nnz_a), dtype=torch.float32, device=dev)
        res = torch.empty(batch, dtype=torch.float32, device=dev) if residual else None
        s = pl.settings
        opts = native.OsqpOptions(max_iter=int(s.max_iter if max_iter is None else max_iter), check_termination=check,
                                  eps_abs=np.float32(s.eps_abs), eps_rel=np.float32(s.eps_rel), warm_start=0,
                                  reuse_factor=1)
        data = native.OsqpAdjointBatch(
            batch=batch, p_values=p.data_ptr(), p_batch=int(p.shape[0]), a_values=a.data_ptr(),
            a_batch=int(a.shape[0]), l=lm.data_ptr(), u=um.data_ptr(), x=x.data_ptr(), z=z.data_ptr(),
            y=y.data_ptr(), dx=dxm.data_ptr(), dy=None if dym is None else dym.data_ptr(), dq=dq.data_ptr(),
            dl=dl.data_ptr(), du=du.data_ptr(), dp=dp.data_ptr(), da=da.data_ptr(),
            adj_prim_res=res.data_ptr() if residual else None,
        )
        native.check(native.lib().wmpc_osqp_adjoint(self.dev.handle, ctypes.byref(opts), ctypes.byref(data), mode_id,
                                                    native.tensor_ptr(ws), wsb, native.current_stream_handle(dev)))
        self.last_adjoint_residual = res
        return dq, dl, du, dp, da


def compile_osqp(
    plan: FixedOSQPPlan,
    dtype=np.float64,
    *,
    qdldl_backend: str = "jax",
    qdldl_factor_backend: str | None = None,
    qdldl_solve_backend: str | None = None,
    transpose_work: bool = False,
    segmented: bool = False,
    segment_budget: int = 64,
    segment_strategy: str = "optimal",
    level_scheduled_solve: bool = False,
    level_scheduled_solve_threshold: int = 1,
    derivatives: bool = False,
    derivative_refinement_iters: int = 100,
    mode: str = "persistent",
    device=None,
    adjoint_iters: int | None = None,
    schedule: dict | None = None,
) -> CompiledOSQP:
    """Compile fixed-pattern batched OSQP iterations (solver.py:685-1492).

    ``derivatives=True`` adds the reverse-mode callables (``solve_xy``,
    ``solve_primal``, and ``solve``/``solve_warm_start`` with gradients) on the
    adjoint that re-uses the forward factor; ``adjoint_iters`` sets its ADMM
    iterations (default ``settings.max_iter``).  ``derivative_refinement_iters``
    is accepted for signature compatibility (the reference's refinement of a
    separately factored adjoint system does not exist here).  ``schedule``:
    streaming-schedule knobs for this problem (``autotune.KNOBS`` names, e.g.
    the ``best`` of ``autotune_stream``), fixed when the problem is created.
    """

    import torch

    if schedule:
        from .autotune import apply

        with apply(schedule):
            return compile_osqp(plan, dtype, qdldl_backend=qdldl_backend, qdldl_factor_backend=qdldl_factor_backend,
                                qdldl_solve_backend=qdldl_solve_backend, transpose_work=transpose_work,
                                segmented=segmented, segment_budget=segment_budget, segment_strategy=segment_strategy,
                                level_scheduled_solve=level_scheduled_solve,
                                level_scheduled_solve_threshold=level_scheduled_solve_threshold,
                                derivatives=derivatives, derivative_refinement_iters=derivative_refinement_iters,
                                mode=mode, device=device, adjoint_iters=adjoint_iters)

    qdldl = compile_qdldl_variant(
        plan.qdldl_plan,
        dtype=dtype,
        backend=qdldl_backend,
        factor_backend=qdldl_factor_backend,
        solve_backend=qdldl_solve_backend,
        transpose_work=transpose_work,
        segmented=segmented,
        segment_budget=segment_budget,
        segment_strategy=segment_strategy,
        level_scheduled_solve=level_scheduled_solve,
        level_scheduled_solve_threshold=level_scheduled_solve_threshold,
        device=device,
    )
    engine = OSQPEngine(plan, device=device, mode=mode, kkt_plan=qdldl.device_plan)
    settings = plan.settings
    dev = engine.device

    def factor(p_values, a_values):
        return engine.factor(p_values, a_values)

    def solve(p_values, a_values, q, l, u):
        return engine.solve(p_values, a_values, q, l, u)

    def solve_warm_start(p_values, a_values, q, l, u, warm_start_x, warm_start_z, warm_start_y):
        return engine.solve(p_values, a_values, q, l, u, warm=(warm_start_x, warm_start_z, warm_start_y))

    def solve_with_factor(lx, dinv, p_values, a_values, q, l, u):
        return engine.solve(p_values, a_values, q, l, u, factor=(lx, dinv))

    def solve_with_factor_warm_start(lx, dinv, p_values, a_values, q, l, u, warm_start_x, warm_start_z, warm_start_y):
        return engine.solve(p_values, a_values, q, l, u, warm=(warm_start_x, warm_start_z, warm_start_y),
                            factor=(lx, dinv))

    def linear_solve_loop(lx, dinv, rhs):
        sol = rhs_for_compiled_qdldl(qdldl, _as_f32(rhs, dev, "rhs")).contiguous()
        for _ in range(settings.max_iter):
            sol = qdldl.solve(lx, dinv, sol)
        return batch_from_compiled_qdldl(qdldl, sol)

    def init_warm_start(batch_size: int) -> OSQPWarmStart:
        return OSQPWarmStart(
            x=torch.zeros((batch_size, plan.n), dtype=torch.float32, device=dev),
            z=torch.zeros((batch_size, plan.m), dtype=torch.float32, device=dev),
            y=torch.zeros((batch_size, plan.m), dtype=torch.float32, device=dev),
        )

    extra = {}
    if derivatives:
        from .adjoint import make_derivative_callables

        extra = make_derivative_callables(plan, engine, adjoint_iters)

    return CompiledOSQP(
        plan=plan,
        settings=settings,
        qdldl=qdldl,
        solve=extra.get("solve", solve),
        factor=factor,
        solve_with_factor=solve_with_factor,
        variant=qdldl.variant + f"+{mode}",
        dtype=qdldl.dtype,
        linear_solve_loop=linear_solve_loop,
        init_warm_start=init_warm_start,
        solve_warm_start=extra.get("solve_warm_start", solve_warm_start),
        solve_with_factor_warm_start=solve_with_factor_warm_start,
        adjoint_derivative_compute=extra.get("adjoint_derivative_compute"),
        adjoint_derivative_get_mat=extra.get("adjoint_derivative_get_mat"),
        adjoint_derivative_get_vec=extra.get("adjoint_derivative_get_vec"),
        solve_primal=extra.get("solve_primal"),
        solve_xy=extra.get("solve_xy"),
        engine=engine,
    )


def solve_classes(problems_, max_iter=None, check_termination=None):
    """Several problem classes (one OSQP engine each, persistent mode, one
    device) solved by one persistent launch: ``problems_`` is a sequence of
    ``(engine, p_values, a_values, q, l, u, warm)`` (``warm`` None or
    ``(x, z, y)``); returns one ``(x, z, y, prim_res, dual_res, obj_val, iters,
    status)`` per class.  The work-queue form of ``engine.solve`` for a
    mixed-size batch (``wmpc_osqp_solve_persistent``)."""
    lib = native.lib()
    n = len(problems_)
    if not 1 <= n <= 6:
        raise ValueError("1 to 6 classes per launch")
    datas, optss, keeps, outs, wss = [], [], [], [], []
    dev = None
    for engine, p, a, q, l, u, warm in problems_:
        if engine.mode != "persistent":
            raise ValueError("every class needs a persistent-mode engine")
        if dev is None:
            dev = engine.device
        elif engine.device != dev:
            raise ValueError("every class must be on one device")
        data, opts, keep, out, batch = engine._batch_args(p, a, q, l, u, warm, max_iter, check_termination, None)
        ws, wsb = _workspace(lib.wmpc_osqp_workspace_bytes(engine.dev.handle, batch, _MODES["persistent"], 0), dev)
        datas.append(data)
        optss.append(opts)
        keeps.append(keep)
        outs.append(out)
        wss.append((ws, wsb))
    handles = (ctypes.c_void_p * n)(*[e.dev.handle for e, *_ in problems_])
    opts_arr = (native.OsqpOptions * n)(*optss)
    data_arr = (native.OsqpBatch * n)(*datas)
    ws_arr = (ctypes.c_void_p * n)(*[native.tensor_ptr(w) for w, _ in wss])
    wsb_arr = (ctypes.c_size_t * n)(*[b for _, b in wss])
    native.check(lib.wmpc_osqp_solve_persistent(handles, opts_arr, data_arr, n, ws_arr, wsb_arr,
                                                native.current_stream_handle(dev)))
    return outs
