"""ctypes binding of ``libwarpmpc_b200.so`` (the C ABI in include/warpmpc_b200.h).

There is no fallback: if the library cannot be loaded, every call raises.
Tensors are ``torch`` CUDA tensors; their raw device pointers and the current
torch CUDA stream are handed to the library.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import threading

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "libwarpmpc_b200.so"

WMPC_OK = 0
WMPC_ERR_INVALID_ARGUMENT = 1
WMPC_ERR_CUDA = 2
WMPC_ERR_UNSUPPORTED = 3
WMPC_ERR_WORKSPACE = 4
WMPC_ERR_OUT_OF_MEMORY = 5

WMPC_OSQP_PLAIN = 0
WMPC_OSQP_PERSISTENT = 1

STATUS_MAX_ITER = 0
STATUS_SOLVED = 1
STATUS_NONFINITE = 2
STATUS_ZERO_PIVOT = 4
STATUS_KERNEL_ABORT = 8

_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)


class PatternDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("nnz_a", ctypes.c_int32),
        ("nnz_l", ctypes.c_int32),
        ("perm_to_orig", _i32p),
        ("diag_pos", _i32p),
        ("init_ptr", _i32p),
        ("init_rows", _i32p),
        ("init_pos", _i32p),
        ("proc_ptr", _i32p),
        ("proc_cols", _i32p),
        ("proc_lidx", _i32p),
        ("proc_offsets", _i32p),
        ("lp", _i32p),
        ("li", _i32p),
        ("p", _i32p),
        ("pinv", _i32p),
    ]


class QuadrotorModel(ctypes.Structure):
    """wmpc_quadrotor_model: the rigid-body model's constants."""

    _fields_ = [(k, ctypes.c_float) for k in ("mass", "jx", "jy", "jz", "arm", "yaw_coef", "gravity")]


class OsqpDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("m", ctypes.c_int32),
        ("nnz_p", ctypes.c_int32),
        ("nnz_a", ctypes.c_int32),
        ("nnz_kkt", ctypes.c_int32),
        ("sigma", ctypes.c_float),
        ("alpha", ctypes.c_float),
        ("kkt_base", _f32p),
        ("p_to_kkt", _i32p),
        ("p_diag_sigma", _f32p),
        ("a_to_kkt", _i32p),
        ("p_scale", _f32p),
        ("a_scale", _f32p),
        ("a_rows", _i32p),
        ("a_cols", _i32p),
        ("p_full_rows", _i32p),
        ("p_full_cols", _i32p),
        ("p_full_value_map", _i32p),
        ("nnz_p_full", ctypes.c_int32),
        ("rho_vec", _f32p),
        ("rho_inv_vec", _f32p),
        ("q_scale", _f32p),
        ("scaling_d", _f32p),
        ("scaling_dinv", _f32p),
        ("scaling_e", _f32p),
        ("scaling_einv", _f32p),
        ("y_scale", _f32p),
        ("y_unscale", _f32p),
        ("rho_type", _i32p),
        ("rho_to_kkt", _i32p),
        ("rho", ctypes.c_float),
    ]


class OsqpOptions(ctypes.Structure):
    _fields_ = [
        ("max_iter", ctypes.c_int32),
        ("check_termination", ctypes.c_int32),
        ("eps_abs", ctypes.c_float),
        ("eps_rel", ctypes.c_float),
        ("warm_start", ctypes.c_int32),
        ("reuse_factor", ctypes.c_int32),
        ("adaptive_rho_interval", ctypes.c_int32),
        ("adaptive_rho_tolerance", ctypes.c_float),
    ]


class OsqpAdjointBatch(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int32),
        ("p_values", ctypes.c_void_p),
        ("p_batch", ctypes.c_int32),
        ("a_values", ctypes.c_void_p),
        ("a_batch", ctypes.c_int32),
        ("l", ctypes.c_void_p),
        ("u", ctypes.c_void_p),
        ("x", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("dx", ctypes.c_void_p),
        ("dy", ctypes.c_void_p),
        ("dq", ctypes.c_void_p),
        ("dl", ctypes.c_void_p),
        ("du", ctypes.c_void_p),
        ("dp", ctypes.c_void_p),
        ("da", ctypes.c_void_p),
        ("adj_prim_res", ctypes.c_void_p),
    ]


class OsqpBatch(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int32),
        ("p_values", ctypes.c_void_p),
        ("p_batch", ctypes.c_int32),
        ("a_values", ctypes.c_void_p),
        ("a_batch", ctypes.c_int32),
        ("q", ctypes.c_void_p),
        ("l", ctypes.c_void_p),
        ("u", ctypes.c_void_p),
        ("x0", ctypes.c_void_p),
        ("z0", ctypes.c_void_p),
        ("y0", ctypes.c_void_p),
        ("x", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("prim_res", ctypes.c_void_p),
        ("dual_res", ctypes.c_void_p),
        ("obj", ctypes.c_void_p),
        ("iters", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("rho", ctypes.c_void_p),
        ("rho_updates", ctypes.c_void_p),
    ]


class LineSearchSettings(ctypes.Structure):
    _fields_ = [
        ("g_max", ctypes.c_float),
        ("g_min", ctypes.c_float),
        ("gamma_c", ctypes.c_float),
        ("armijo_factor", ctypes.c_float),
        ("constraint_scale", ctypes.c_float),
        ("cost_accept_uses_trial_cost", ctypes.c_int32),
    ]


class SqpStepBatch(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("m", ctypes.c_int32),
        ("n_steps", ctypes.c_int32),
        ("n_candidates", ctypes.c_int32),
        ("step_lengths", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("direction", ctypes.c_void_p),
        ("q", ctypes.c_void_p),
        ("constraint_l", ctypes.c_void_p),
        ("g", ctypes.c_void_p),
        ("constraint_u", ctypes.c_void_p),
        ("baseline_cost", ctypes.c_void_p),
        ("candidate_costs", ctypes.c_void_p),
        ("candidate_violations", ctypes.c_void_p),
        ("z_next", ctypes.c_void_p),
        ("step_length", ctypes.c_void_p),
        ("cost", ctypes.c_void_p),
        ("violation", ctypes.c_void_p),
        ("baseline_violation", ctypes.c_void_p),
        ("reason", ctypes.c_void_p),
        ("accepted", ctypes.c_void_p),
        ("is_finite", ctypes.c_void_p),
        ("candidate_acceptance", ctypes.c_void_p),
    ]


class SqpAssembleDims(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("batch", "n", "nnz_p", "nnz_a", "m", "n_stages", "width")]


# (name, restype, argtypes) of every exported symbol; also used by the
# symbol-export test.
SIGNATURES = {
    "wmpc_plan_create": (ctypes.c_int, [ctypes.POINTER(PatternDesc), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "wmpc_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "wmpc_plan_info": (ctypes.c_int, [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p, _i32p]),
    "wmpc_factor_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int32]),
    "wmpc_solve_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int32]),
    "wmpc_factor": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "wmpc_solve": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "wmpc_solve_noalloc": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_int32, ctypes.c_void_p],
    ),
    "wmpc_factor_solve": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t,
         ctypes.c_void_p],
    ),
    "wmpc_osqp_create": (ctypes.c_int, [ctypes.POINTER(OsqpDesc), ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "wmpc_osqp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "wmpc_osqp_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "wmpc_osqp_stream_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "wmpc_osqp_factor": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "wmpc_osqp_solve": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(OsqpOptions), ctypes.POINTER(OsqpBatch), ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "wmpc_osqp_adjoint_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "wmpc_osqp_adjoint": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(OsqpOptions), ctypes.POINTER(OsqpAdjointBatch), ctypes.c_int32,
         ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "wmpc_osqp_solve_persistent": (
        ctypes.c_int,
        [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(OsqpOptions), ctypes.POINTER(OsqpBatch), ctypes.c_int32,
         ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p],
    ),
    "wmpc_quadrotor_rk4": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "wmpc_quadrotor_jac_pattern": (ctypes.c_int, [_i32p, _i32p]),
    "wmpc_solve_tables_host": (ctypes.c_int, [ctypes.POINTER(PatternDesc), _i32p, ctypes.c_int64,
                                              ctypes.POINTER(ctypes.c_int64)]),
    "wmpc_stream_schedule_host": (
        ctypes.c_int,
        [ctypes.POINTER(PatternDesc), _f32p, _f32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
         ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)],
    ),
    "wmpc_constraint_violation": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "wmpc_filter_line_search": (
        ctypes.c_int,
        [ctypes.POINTER(LineSearchSettings), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "wmpc_sqp_line_search_step": (
        ctypes.c_int, [ctypes.POINTER(LineSearchSettings), ctypes.POINTER(SqpStepBatch), ctypes.c_void_p]
    ),
    "wmpc_sym_matvec": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p],
    ),
    "wmpc_sqp_assemble": (
        ctypes.c_int,
        [ctypes.POINTER(SqpAssembleDims)] + [ctypes.c_void_p] * 14 + [ctypes.c_void_p],
    ),
    "wmpc_profile_begin": (ctypes.c_int, []),
    "wmpc_profile_select": (ctypes.c_int, [ctypes.c_int32]),
    "wmpc_stream_last_launch": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "wmpc_profile_end": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), _i32p, ctypes.POINTER(ctypes.c_int64)]),
    "wmpc_launch_count": (ctypes.c_int64, []),
    "wmpc_last_error_string": (ctypes.c_char_p, []),
    "wmpc_version": (ctypes.c_char_p, []),
}

_lib = None
_lock = threading.Lock()


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"warpmpc_b200 native error {code}: {message}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load (once) and return the library; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m warpmpc_b200.build` "
                    "(there is no CPU fallback)"
                )
            handle = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(code: int) -> None:
    if code != WMPC_OK:
        msg = lib().wmpc_last_error_string().decode("utf-8", "replace")
        if code == WMPC_ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        if code == WMPC_ERR_UNSUPPORTED:
            raise NotImplementedError(msg)
        raise NativeError(code, msg)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def ptr_i32(a: np.ndarray):
    return a.ctypes.data_as(_i32p)


def ptr_f32(a: np.ndarray):
    return a.ctypes.data_as(_f32p)


def tensor_ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def current_stream_handle(device) -> int:
    import torch

    return int(torch.cuda.current_stream(device).cuda_stream)


def device_index(device) -> int:
    import torch

    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError("warpmpc_b200 runs on CUDA devices only")
    return torch.cuda.current_device() if dev.index is None else dev.index


def require_cuda() -> None:
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("warpmpc_b200 needs a CUDA device (there is no CPU fallback)")


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)


def loaded_library_path() -> str:
    lib()
    return str(LIB_PATH)


def version() -> str:
    return lib().wmpc_version().decode()


def env_flag(name: str, default: str = "0") -> bool:
    return os.environ.get(name, default) not in ("0", "", "false", "False")


PROFILE_DOMINANT = 0
PROFILE_FACTOR = 1


def profile_begin(channel: int = PROFILE_DOMINANT) -> None:
    """Start timing the launches of one channel: the dominant kernel (0) or
    the factorization kernels (1)."""
    check(lib().wmpc_profile_select(channel))
    check(lib().wmpc_profile_begin())


def profile_end() -> tuple[float, int, int]:
    """(dominant kernel ms summed, dominant launches, all launches) since profile_begin."""
    ms = ctypes.c_float()
    n = ctypes.c_int32()
    total = ctypes.c_int64()
    check(lib().wmpc_profile_end(ctypes.byref(ms), ctypes.byref(n), ctypes.byref(total)))
    check(lib().wmpc_profile_select(PROFILE_DOMINANT))
    return float(ms.value), int(n.value), int(total.value)


def stream_last_launch() -> dict:
    """The last streaming ADMM launch: schedule form, CTAs per SM, grid, shared memory."""
    info = (ctypes.c_int32 * 4)()
    check(lib().wmpc_stream_last_launch(info))
    return {"form": {0: None, 1: "plain", 2: "frontier"}.get(int(info[0])), "ctas_per_sm": int(info[1]),
            "grid": int(info[2]), "smem_bytes": int(info[3])}
