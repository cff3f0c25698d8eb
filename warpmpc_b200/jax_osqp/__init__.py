"""Fixed-pattern batched OSQP with a CUDA backend.

Mirror of ``warpmpc.jax_osqp`` (``warpmpc/jax_osqp/__init__.py``).
"""

from .planning import build_osqp_plan
from .types import CompiledOSQP, FixedOSQPPlan, OSQPDerivativePlan, OSQPSettings, OSQPWarmStart


def __getattr__(name):
    if name in ("compile_osqp", "solve_classes", "values_for_compiled_qdldl", "rhs_for_compiled_qdldl",
                "batch_from_compiled_qdldl"):
        from . import solver

        return getattr(solver, name)
    raise AttributeError(name)


__all__ = [
    "CompiledOSQP",
    "FixedOSQPPlan",
    "OSQPDerivativePlan",
    "OSQPSettings",
    "OSQPWarmStart",
    "batch_from_compiled_qdldl",
    "build_osqp_plan",
    "compile_osqp",
    "rhs_for_compiled_qdldl",
    "solve_classes",
    "values_for_compiled_qdldl",
]
