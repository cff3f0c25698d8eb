"""Compiled batched LDL^T factor/solve on the CUDA library.

Mirror of ``compile_qdldl`` / ``compile_qdldl_variant``
(``warpmpc/jax_qdldl/core.py:314-317, 544-1051``) with the backend name
``"cuda"`` added next to the reference's ``"jax"``/``"warp"``
(``_normalize_backend_name`` 513-516, dispatch 638-652).  The compiled
callables take and return ``torch`` CUDA tensors in the Warp backend's
symbolic-major layouts (``values_layout="original_symbolic"``,
``rhs_layout="symbolic"``): ``values (nnz_a, B)``, ``rhs (n, B)``.

The reference's variant knobs (``segmented``, ``segment_budget``,
``segment_strategy``, ``level_scheduled_solve``,
``level_scheduled_solve_threshold``) are validated exactly as the reference
validates them and recorded in the variant name; the CUDA kernels walk ragged
tables, so padded-loop segmentation and level launches have no work to save.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import native
from .planning import _make_segment_arrays, plan_ragged_program
from .types import CompiledQDLDL, QDLDLPlan

_KNOWN_BACKENDS = {"jax", "warp", "cuda"}


def _normalize_backend_name(name: str, *, role: str) -> str:
    if name not in _KNOWN_BACKENDS:
        raise ValueError(f"unknown QDLDL {role} backend {name!r}")
    return name


class DevicePlan:
    """A plan's pattern tables uploaded to one CUDA device (``wmpc_plan``)."""

    def __init__(self, plan: QDLDLPlan, device=None):
        native.require_cuda()
        self.plan = plan
        self.device_index = native.device_index(device if device is not None else "cuda")
        rg = plan_ragged_program(plan)
        arrays = {
            "perm_to_orig": native.i32(plan.perm_to_orig),
            "diag_pos": native.i32(plan.diag_pos),
            "init_ptr": native.i32(rg["init_ptr"]),
            "init_rows": native.i32(rg["init_rows"]),
            "init_pos": native.i32(rg["init_pos"]),
            "proc_ptr": native.i32(rg["proc_ptr"]),
            "proc_cols": native.i32(rg["proc_cols"]),
            "proc_lidx": native.i32(rg["proc_lidx"]),
            "proc_offsets": native.i32(rg["proc_offsets"]),
            "lp": native.i32(plan.lp),
            "li": native.i32(plan.li),
            "p": native.i32(plan.p),
            "pinv": native.i32(plan.pinv),
        }
        desc = native.PatternDesc(n=plan.n, nnz_a=plan.nnz_a, nnz_l=plan.nnz_l,
                                  **{k: native.ptr_i32(v) for k, v in arrays.items()})
        handle = ctypes.c_void_p()
        native.check(native.lib().wmpc_plan_create(ctypes.byref(desc), self.device_index, ctypes.byref(handle)))
        self.handle = handle

    @property
    def torch_device(self):
        import torch

        return torch.device("cuda", self.device_index)

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                native.lib().wmpc_plan_destroy(handle)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = None


def _workspace(nbytes: int, device):
    import torch

    if nbytes <= 0:
        return None, 0
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device), int(nbytes)


def _as_f32(t, device, name: str):
    import torch

    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.asarray(t, dtype=np.float32))
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32 (the CUDA backend computes in float32), got {t.dtype}")
    return t.to(device).contiguous()


def compile_qdldl_cuda(
    plan: QDLDLPlan,
    dtype=np.float32,
    *,
    transpose_work: bool = True,
    segmented: bool = False,
    segment_budget: int = 64,
    segment_strategy: str = "optimal",
    level_scheduled_solve: bool = False,
    level_scheduled_solve_threshold: int = 1,
    device=None,
) -> CompiledQDLDL:
    """CUDA-backed fixed-pattern factor/solve (symbolic-major layouts)."""

    import torch

    dtype = np.dtype(dtype)
    if dtype != np.dtype(np.float32):
        raise ValueError("the CUDA QDLDL backend computes in float32")
    if level_scheduled_solve_threshold < 1:
        raise ValueError("level_scheduled_solve_threshold must be at least 1")
    segments = None
    if segmented:
        segments = {
            "process": _make_segment_arrays(plan.process_mask, segment_budget=segment_budget, segment_strategy=segment_strategy),
            "col": _make_segment_arrays(plan.col_mask, segment_budget=segment_budget, segment_strategy=segment_strategy),
        }
    dplan = DevicePlan(plan, device)
    dev = dplan.torch_device
    lib = native.lib()
    n, nnz_a, nnz_l = plan.n, plan.nnz_a, plan.nnz_l

    def factor(a_values):
        vals = _as_f32(a_values, dev, "a_values")
        if vals.dim() != 2 or vals.shape[0] != nnz_a:
            raise ValueError(f"a_values must have shape ({nnz_a}, batch)")
        batch = int(vals.shape[1])
        lx = torch.empty((nnz_l, batch), dtype=torch.float32, device=dev)
        d = torch.empty((n, batch), dtype=torch.float32, device=dev)
        dinv = torch.empty((n, batch), dtype=torch.float32, device=dev)
        ws, wsb = _workspace(lib.wmpc_factor_workspace_bytes(dplan.handle, batch), dev)
        native.check(lib.wmpc_factor(dplan.handle, vals.data_ptr(), batch, 1, lx.data_ptr(), d.data_ptr(),
                                     dinv.data_ptr(), batch, native.tensor_ptr(ws), wsb,
                                     native.current_stream_handle(dev)))
        return lx, d, dinv

    def solve(lx, dinv, rhs):
        lx = _as_f32(lx, dev, "lx")
        dinv = _as_f32(dinv, dev, "dinv")
        rhs = _as_f32(rhs, dev, "rhs")
        if rhs.dim() != 2 or rhs.shape[0] != n:
            raise ValueError(f"rhs must have shape ({n}, batch)")
        batch = int(rhs.shape[1])
        fb = int(lx.shape[1])
        if lx.shape[0] != nnz_l or dinv.shape != (n, fb) or fb not in (1, batch):
            raise ValueError("lx/dinv shapes do not match the plan or the rhs batch")
        out = torch.empty((n, batch), dtype=torch.float32, device=dev)
        ws, wsb = _workspace(lib.wmpc_solve_workspace_bytes(dplan.handle, batch), dev)
        native.check(lib.wmpc_solve(dplan.handle, lx.data_ptr(), dinv.data_ptr(), 1 if fb > 1 else 0,
                                    rhs.data_ptr(), out.data_ptr(), batch, native.tensor_ptr(ws), wsb,
                                    native.current_stream_handle(dev)))
        return out

    def factor_and_solve(a_values, rhs):
        lx, d, dinv = factor(a_values)
        return solve(lx, dinv, rhs), lx, d

    variant = ["cuda"]
    if transpose_work:
        variant.append("transpose")
    if segmented:
        variant += ["segmented", f"budget{segment_budget}", segment_strategy]
    if level_scheduled_solve:
        variant.append("levelsolve")
        if level_scheduled_solve_threshold != 1:
            variant.append(f"threshold{level_scheduled_solve_threshold}")
    compiled = CompiledQDLDL(
        plan=plan,
        dtype=dtype,
        factor=factor,
        solve=solve,
        factor_and_solve=factor_and_solve,
        variant="+".join(variant),
        values_layout="original_symbolic",
        rhs_layout="symbolic",
        backend="cuda",
        factor_backend="cuda",
        solve_backend="cuda",
        device_plan=dplan,
    )
    object.__setattr__(compiled, "_segments", segments)
    return compiled


def compile_qdldl_variant(
    plan: QDLDLPlan,
    dtype=np.float64,
    *,
    backend: str = "jax",
    factor_backend: str | None = None,
    solve_backend: str | None = None,
    transpose_work: bool = False,
    segmented: bool = False,
    segment_budget: int = 64,
    segment_strategy: str = "optimal",
    level_scheduled_solve: bool = False,
    level_scheduled_solve_threshold: int = 1,
    device=None,
) -> CompiledQDLDL:
    """Compile a fixed-pattern LDL^T variant (core.py:544-1051).

    Only ``backend="cuda"`` is implemented by this package; ``"jax"`` and
    ``"warp"`` are the reference's own backends and raise ``ImportError``
    here (their runtimes are not part of this package).
    """

    factor_backend = backend if factor_backend is None else factor_backend
    solve_backend = backend if solve_backend is None else solve_backend
    factor_backend = _normalize_backend_name(factor_backend, role="factor")
    solve_backend = _normalize_backend_name(solve_backend, role="solve")
    for name in (factor_backend, solve_backend):
        if name != "cuda":
            raise ImportError(
                f"QDLDL backend {name!r} is provided by the reference package (warpmpc); "
                "warpmpc_b200 implements backend='cuda'"
            )
    return compile_qdldl_cuda(
        plan,
        dtype=dtype,
        transpose_work=transpose_work,
        segmented=segmented,
        segment_budget=segment_budget,
        segment_strategy=segment_strategy,
        level_scheduled_solve=level_scheduled_solve,
        level_scheduled_solve_threshold=level_scheduled_solve_threshold,
        device=device,
    )


def compile_qdldl(plan: QDLDLPlan, dtype=np.float32, *, device=None) -> CompiledQDLDL:
    """Compile the default CUDA variant for ``plan`` (core.py:314-317)."""
    return compile_qdldl_variant(plan, dtype=dtype, backend="cuda", device=device)
