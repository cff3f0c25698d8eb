"""CPU restatement of the rigid-body quadrotor model of the nonlinear SQP workload.

TEST INFRASTRUCTURE ONLY (oracle): the float64 truth the CUDA model kernel
(``wmpc_quadrotor_rk4``) is checked against, and central finite differences
of it for the kernel's forward-mode Jacobians.

The reference's SQP problems take their stage functions from CasADi
(``warpmpc/jax_sqp/casadi_stage.py:66-189``; its Crazyflie problem in
``benchmarks/problems/crazyflie_sqp.py:56-117`` uses Euler-angle rigid-body
dynamics with an explicit Euler step and the cost Hessian as the QP's P,
``casadi_stage.py:119``).  CasADi is absent here, so this workload's model is
written by hand from the standard rigid-body equations:

state ``x = [p (3), eta = (roll, pitch, yaw) (3), v (3, world frame),
w (3, body rates)]``, input ``u = [f1, f2, f3, f4]`` motor thrusts (N),

    p'   = v
    eta' = W(eta) w          (Euler-angle rate map, ZYX angles)
    v'   = (f1+f2+f3+f4)/m R(eta) e3 - g e3
    w'   = J^-1 (tau - w x J w)
    tau  = (d (-f1 - f2 + f3 + f4), d (-f1 + f2 + f3 - f4), k (-f1 + f2 - f3 + f4))

with m = 0.03 kg, J = diag(1.4e-5, 1.4e-5, 2.2e-5) kg m^2, arm d = 0.046/sqrt(2)
m (X configuration), yaw torque coefficient k = 0.006 m, g = 9.81, and the
classical fourth-order Runge-Kutta step with dt = 0.02 s.
"""

from __future__ import annotations

import numpy as np

MASS = 0.03
INERTIA = np.array([1.4e-5, 1.4e-5, 2.2e-5])
ARM = 0.046 / np.sqrt(2.0)
YAW_COEF = 0.006
GRAVITY = 9.81
DT = 0.02
U_MAX = 0.15
U_HOVER = MASS * GRAVITY / 4.0
NX, NU = 12, 4


def continuous(x, u):
    """x' for states x (..., 12) and inputs u (..., 4)."""
    phi, theta, psi = x[..., 3], x[..., 4], x[..., 5]
    v = x[..., 6:9]
    wx, wy, wz = x[..., 9], x[..., 10], x[..., 11]
    f1, f2, f3, f4 = u[..., 0], u[..., 1], u[..., 2], u[..., 3]
    thrust = f1 + f2 + f3 + f4
    cphi, sphi = np.cos(phi), np.sin(phi)
    cth, sth = np.cos(theta), np.sin(theta)
    cpsi, spsi = np.cos(psi), np.sin(psi)
    tth = sth / cth
    # body z axis in the world frame (third column of R = Rz(psi) Ry(theta) Rx(phi))
    r13 = cpsi * sth * cphi + spsi * sphi
    r23 = spsi * sth * cphi - cpsi * sphi
    r33 = cth * cphi
    a = thrust / MASS
    dphi = wx + sphi * tth * wy + cphi * tth * wz
    dth = cphi * wy - sphi * wz
    dpsi = (sphi * wy + cphi * wz) / cth
    tx = ARM * (-f1 - f2 + f3 + f4)
    ty = ARM * (-f1 + f2 + f3 - f4)
    tz = YAW_COEF * (-f1 + f2 - f3 + f4)
    jx, jy, jz = INERTIA
    dwx = (tx - (jz - jy) * wy * wz) / jx
    dwy = (ty - (jx - jz) * wx * wz) / jy
    dwz = (tz - (jy - jx) * wx * wy) / jz
    return np.stack([v[..., 0], v[..., 1], v[..., 2], dphi, dth, dpsi, a * r13, a * r23, a * r33 - GRAVITY,
                     dwx, dwy, dwz], axis=-1)


def rk4(x, u, dt=DT):
    """One classical Runge-Kutta step of the model."""
    k1 = continuous(x, u)
    k2 = continuous(x + 0.5 * dt * k1, u)
    k3 = continuous(x + 0.5 * dt * k2, u)
    k4 = continuous(x + dt * k3, u)
    return x + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)


def rk4_jacobian_fd(x, u, h=1e-6):
    """Central differences of rk4 w.r.t. [x, u]: (..., 12, 16)."""
    z = np.concatenate([x, u], axis=-1)
    out = np.empty(z.shape[:-1] + (NX, NX + NU))
    for c in range(NX + NU):
        zp, zm = z.copy(), z.copy()
        zp[..., c] += h
        zm[..., c] -= h
        out[..., :, c] = (rk4(zp[..., :NX], zp[..., NX:]) - rk4(zm[..., :NX], zm[..., NX:])) / (2 * h)
    return out


def structural_mask(samples=64, seed=0):
    """(12, 16) boolean: the entries of the RK4 Jacobian that are nonzero at
    generic points (the fixed sparsity of the dynamics rows)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5, 0.5, (samples, NX))
    u = rng.uniform(0.0, U_MAX, (samples, NU))
    j = rk4_jacobian_fd(x, u)
    return np.any(np.abs(j) > 1e-9, axis=0)
