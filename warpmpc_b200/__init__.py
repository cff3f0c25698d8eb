"""warpmpc_b200: B200-native batched fixed-pattern OSQP / QDLDL (LDL^T) solver.

Drop-in ``qdldl_backend="cuda"`` for WarpMPC's batched QP hot path:

* :mod:`warpmpc_b200.jax_qdldl` -- host symbolic planning and the compiled
  batched LDL^T factor/solve (mirror of ``warpmpc.jax_qdldl``);
* :mod:`warpmpc_b200.jax_osqp` -- OSQP plan and the compiled batched ADMM
  solver (mirror of ``warpmpc.jax_osqp``);
* :mod:`warpmpc_b200.native` -- the C-ABI shared library (sm_100a kernels).
"""

__version__ = "0.1.0"
