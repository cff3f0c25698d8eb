"""Batched SQP QP assembly on the GPU (wmpc_sqp_assemble) against the oracle.

Every output entry sums its stage values in stage order from zero, one
float32 addition each, as the oracle does: bit-exact.
"""

import numpy as np
import pytest

from oracle import assembly_ref
from warpmpc_b200 import problems, sqp_problems
from warpmpc_b200.jax_sqp import QPAssembler, build_sparse_mpc_plan

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cls,batch", [(problems.SMALL, 300),
                                       (problems.MPCClass("q5", 12, 4, 5, 10.0, 2.0, 1.0, "quadrotor"), 77),
                                       (problems.MPCClass("q120", 12, 4, 120, 10.0, 2.0, 1.0, "quadrotor"), 5)],
                         ids=["small", "quadrotor_n5", "quadrotor_n120"])
def test_assembly_bitexact(cuda_device, cls, batch):
    import torch

    prob = sqp_problems.make_problem(cls)
    plan = build_sparse_mpc_plan(prob)
    data = sqp_problems.make_data(cls, batch, seed=4)
    gen = torch.Generator(device=cuda_device).manual_seed(1)
    z = torch.randn(batch, int(plan.z_offsets[-1]), device=cuda_device, generator=gen)
    p = torch.randn(batch, cls.nx, device=cuda_device, generator=gen)
    vals = sqp_problems.evaluate_stages(prob, data, z, p)
    asm = QPAssembler(plan, prob)
    got = asm.assemble(asm.pack(vals))
    want = assembly_ref.assemble(plan, prob, [[v.cpu().numpy() for v in s] for s in vals])
    for name, g_, w in zip(got._fields, got, want):
        np.testing.assert_array_equal(g_.cpu().numpy(), w, err_msg=name)


def test_assembled_qp_solves_like_the_oracle(cuda_device):
    """The assembled QP goes straight into the CUDA OSQP solve of the plan's
    OSQP plan: same iterates as the float32 oracle solve of the same data."""
    import torch

    from oracle import osqp_ref
    from warpmpc_b200.jax_osqp import compile_osqp

    cls = problems.SMALL
    prob = sqp_problems.make_problem(cls)
    plan = build_sparse_mpc_plan(prob)
    data = sqp_problems.make_data(cls, 64, seed=5)
    z = torch.zeros(64, int(plan.z_offsets[-1]), device=cuda_device)
    p = torch.rand(64, cls.nx, device=cuda_device) * 2 - 1
    asm = QPAssembler(plan, prob)
    lin = asm.assemble(asm.pack(sqp_problems.evaluate_stages(prob, data, z, p)))
    comp = compile_osqp(plan.osqp_plan, np.float32, qdldl_backend="cuda", transpose_work=True)
    got = comp.solve(lin.p_values, lin.a_values, lin.q, lin.l, lin.u)
    npy = [t.cpu().numpy() for t in (lin.p_values, lin.a_values, lin.q, lin.l, lin.u)]
    want = osqp_ref.solve(plan.osqp_plan, *npy)
    for name, g_, w in zip(("x", "z", "y"), got[:3], want[:3]):
        np.testing.assert_array_equal(g_.cpu().numpy(), w, err_msg=name)
