"""Placeholder-module import of the reference's NumPy/SciPy planners.

TEST INFRASTRUCTURE ONLY (oracle).  Nothing in the product imports this file.

The reference package (hshose/WarpMPC) imports ``jax`` and ``qdldl`` at module
load time, and neither is installed here.  Its symbolic planners, however, are
pure NumPy/SciPy: ``warpmpc/jax_qdldl/core.py:55-510`` (symmetric permutation,
elimination tree, numeric program, segmentation, level sets),
``warpmpc/jax_qdldl/warp_backend.py:1087-1149`` (level packing/schedule,
segment arrays) and ``warpmpc/jax_osqp/solver.py:64-662`` (scaling, rho
vectors, KKT assembly maps, derivative plan).  This module registers minimal
stand-in modules for ``jax``/``jax.numpy``/``jax.lax``/``qdldl`` so those files
import, then exposes the reference functions unchanged.

``qdldl.Solver`` is the only piece with numeric content: the reference asks it
for the AMD permutation and the L pattern (``core.py:276-293``).  The
stand-in takes the permutation from :data:`PERMUTATION_PROVIDER` (set by the
caller, e.g. our own AMD) and returns the L pattern computed by the
reference's *own* ``_symperm_upper``/``_qdldl_etree``/``_build_numeric_program``
so ``build_qdldl_plan``'s cross-checks pass.  The AMD permutation itself is
therefore not pinned by this import (the qdldl package is absent).

It reads the reference tree at import time, so it only works where a
reference checkout exists and the environment variable
``WARPMPC_REFERENCE_ROOT`` names it (there is no default location); golden
fixtures made with it are committed under ``tests/golden``, and the live
comparisons in the tests skip when the variable is unset.
"""

from __future__ import annotations

import os
import sys
import types

import numpy as np
import scipy.sparse as sp

REFERENCE_ROOT = os.environ.get("WARPMPC_REFERENCE_ROOT", "")

# Callable (upper_csc) -> permutation array.  Set before calling
# build_qdldl_plan / build_osqp_plan through the reference.
PERMUTATION_PROVIDER = None

_loaded = None


def available() -> bool:
    return bool(REFERENCE_ROOT) and os.path.isdir(os.path.join(REFERENCE_ROOT, "warpmpc"))


def _identity_decorator(fn=None, *args, **kwargs):
    if fn is None or not callable(fn):
        return lambda f: f
    return fn


class _CustomVJP:
    def __init__(self, fn, *args, **kwargs):
        self.fn = fn

    def defvjp(self, *args, **kwargs):
        return None

    def __call__(self, *args, **kwargs):
        return self.fn(*args, **kwargs)


def _install_stubs() -> None:
    jax = types.ModuleType("jax")
    jax.jit = _identity_decorator
    jax.custom_vjp = _CustomVJP
    jax.Array = object
    jax.config = types.SimpleNamespace(jax_enable_x64=False, update=lambda *a, **k: None)
    jnp = types.ModuleType("jax.numpy")
    jnp.dtype = np.dtype
    lax = types.ModuleType("jax.lax")
    experimental = types.ModuleType("jax.experimental")
    sparse = types.ModuleType("jax.experimental.sparse")
    sparse.BCOO = object
    experimental.sparse = sparse
    jax.numpy = jnp
    jax.lax = lax
    jax.experimental = experimental
    sys.modules.setdefault("jax", jax)
    sys.modules.setdefault("jax.numpy", jnp)
    sys.modules.setdefault("jax.lax", lax)
    sys.modules.setdefault("jax.experimental", experimental)
    sys.modules.setdefault("jax.experimental.sparse", sparse)

    qdldl = types.ModuleType("qdldl")

    class Solver:  # stand-in for the qdldl binding's Solver (core.py:276-277)
        def __init__(self, a_upper, upper=True):
            if PERMUTATION_PROVIDER is None:
                raise RuntimeError("ref_import.PERMUTATION_PROVIDER is not set")
            self._a = sp.csc_matrix(a_upper)
            self._p = np.asarray(PERMUTATION_PROVIDER(self._a), dtype=np.int32)

        def factors(self):
            core = sys.modules["warpmpc.jax_qdldl.core"]
            p = self._p
            pinv = core._pinv(p)
            ap, ai, _, _ = core._symperm_upper(self._a, pinv)
            n = self._a.shape[0]
            lnz, etree, _ = core._qdldl_etree(n, ap, ai)
            prog = core._build_numeric_program(n, ap, ai, lnz, etree)
            lp = prog["lp"]
            li = prog["li"]
            l_csc = sp.csc_matrix(
                (np.zeros(li.size), li, lp), shape=(n, n)
            )
            return l_csc, np.zeros(n), p

    qdldl.Solver = Solver
    sys.modules.setdefault("qdldl", qdldl)

    # casadi: only named in annotations and stage-compilation code paths the
    # planners do not run (warpmpc/jax_sqp/casadi_stage.py)
    casadi = types.ModuleType("casadi")

    def _casadi_attr(name):
        # module metadata (__file__, __spec__, ...) stays absent, so tools
        # that walk sys.modules (inspect) are not handed a placeholder class
        if name.startswith("__"):
            raise AttributeError(name)
        return type(name, (), {})

    casadi.__getattr__ = _casadi_attr
    sys.modules.setdefault("casadi", casadi)


def load():
    """Return a namespace with the reference modules (core, warp_backend, solver)."""
    global _loaded
    if _loaded is not None:
        return _loaded
    if not available():
        raise RuntimeError(f"reference checkout not found at {REFERENCE_ROOT}")
    _install_stubs()
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    import importlib

    core = importlib.import_module("warpmpc.jax_qdldl.core")
    warp_backend = importlib.import_module("warpmpc.jax_qdldl.warp_backend")
    solver = importlib.import_module("warpmpc.jax_osqp.solver")
    types_mod = importlib.import_module("warpmpc.jax_osqp.types")
    _loaded = types.SimpleNamespace(
        core=core, warp_backend=warp_backend, solver=solver, osqp_types=types_mod
    )
    return _loaded


def load_sqp():
    """The reference's sparse MPC module (warpmpc/jax_sqp/sparse_mpc.py), whose
    plan builder (532-691) is NumPy/SciPy given stage objects."""
    load()
    import importlib

    return importlib.import_module("warpmpc.jax_sqp.sparse_mpc")
