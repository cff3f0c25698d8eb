"""Fixed-pattern batched LDL^T (QDLDL) with a CUDA backend.

Mirror of ``warpmpc.jax_qdldl`` (``warpmpc/jax_qdldl/__init__.py``).
"""

from .planning import build_qdldl_plan
from .types import CompiledQDLDL, QDLDLPlan


def __getattr__(name):
    if name in ("compile_qdldl", "compile_qdldl_variant"):
        from . import core

        return getattr(core, name)
    raise AttributeError(name)


__all__ = [
    "CompiledQDLDL",
    "QDLDLPlan",
    "build_qdldl_plan",
    "compile_qdldl",
    "compile_qdldl_variant",
]
