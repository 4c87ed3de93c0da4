"""Differentiable rollouts (nexdynipc_b200.diff): batched central-difference
Jacobians against closed forms of the implicit-Euler step, the autograd
Function against the Jacobian, and parameter identification.  The CPU tests
step the copies with the oracle; tests/test_gpu_parity.py runs the device
batch."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, diff, scenes
from oracle import refcpu


def oracle_runner(worlds, steps):
    out = []
    for w in worlds:
        ow = refcpu.OracleWorld(w)
        for _ in range(steps):
            ow.step()
        out.append(ow.state())
    return out


def free_body(force=None, vel=(0.3, 1.0, -0.2), mass=2.0):
    sb = scenes.SceneBuilder("free")
    sb.add_body(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (0.0, 1.0, 0.0), mass=mass, inertia=np.eye(3),
                vel=vel)
    if force is not None:
        sb.force_drive(0, force)
    return sb.build(abi.default_settings(), 0.01, 20)


def test_velocity_jacobian_of_a_free_body():
    # implicit Euler under gravity: p_K = p_0 + K dt v_0 + dt^2 g K (K + 1) / 2
    sc = free_body()
    spec = diff.ParamSpec(["velocity"], bodies=[0])
    K = 20
    y, J = diff.rollout_jacobian(sc, spec, spec.get(sc), K, [0], runner=oracle_runner)
    assert np.allclose(J[0:3], K * sc.dt * np.eye(3), rtol=0, atol=1e-8)
    assert np.abs(J[3:7]).max() == 0.0           # no rotation
    v0 = np.array([0.3, 1.0, -0.2])
    p = np.array([0.0, 1.0, 0.0]) + K * sc.dt * v0 + sc.dt ** 2 * np.array([0, -9.81, 0]) * K * (K + 1) / 2
    assert np.allclose(y[0:3], p, rtol=0, atol=1e-10)


def test_mass_jacobian_under_a_force_drive():
    # ForceDriveForm adds F / m to the acceleration: dp_K/dm = -dt^2 F/m^2 K (K+1)/2
    F = np.array([1.0, 3.0, -2.0])
    m = 2.0
    sc = free_body(force=F, mass=m)
    spec = diff.ParamSpec(["mass"], bodies=[0])
    K = 20
    _, J = diff.rollout_jacobian(sc, spec, spec.get(sc), K, [0], runner=oracle_runner)
    expect = -sc.dt ** 2 * F / m ** 2 * K * (K + 1) / 2
    assert np.allclose(J[0:3, 0], expect, rtol=1e-6, atol=1e-10)


def pendulum():
    sb = scenes.SceneBuilder("pendulum")
    e_v, e_f = np.zeros((0, 3)), np.zeros((0, 3), np.int32)
    sb.add_body(e_v, e_f, (0, 0, 0), mass=1.0, inertia=np.eye(3))
    sb.fix(0)
    sb.add_body(e_v, e_f, (0.5, 0, 0), mass=1.0, inertia=0.1 * np.eye(3), vel=(0.0, 0.5, 0.0))
    sb.hinge(0, 1, (0, 0, 0), (-0.5, 0, 0), (0, 0, 1), (0, 0, 1), stiffness=1e6)
    s = abi.default_settings()
    s.alm_max_iters = 6
    return sb.build(s, 0.01, 15)


def test_autograd_function_matches_the_jacobian():
    torch = pytest.importorskip("torch")
    sc = pendulum()
    spec = diff.ParamSpec(["velocity", "mass", "joint_stiffness"], bodies=[1], joints=[1])
    theta0 = spec.get(sc)
    f = diff.rollout_function(sc, spec, 15, [1], runner=oracle_runner)
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    target = torch.zeros(7, dtype=torch.float64)
    loss = ((f(theta) - target) ** 2).sum()
    loss.backward()
    y, J = diff.rollout_jacobian(sc, spec, theta0, 15, [1], runner=oracle_runner)
    assert np.allclose(theta.grad.numpy(), J.T @ (2 * y), rtol=1e-12, atol=1e-14)
    # the chain rule through the Function matches a directional difference of the loss
    d = np.array([0.3, -0.2, 0.1, 0.05, 1e3])
    eps = 1e-4
    lp = float(((diff.rollout(sc, spec, theta0 + eps * d, 15, [1], oracle_runner)) ** 2).sum())
    lm = float(((diff.rollout(sc, spec, theta0 - eps * d, 15, [1], oracle_runner)) ** 2).sum())
    assert abs((lp - lm) / (2 * eps) - theta.grad.numpy() @ d) <= 1e-4 * max(1.0, abs(theta.grad.numpy() @ d))


def test_fit_recovers_initial_velocity():
    # identify the pendulum link's initial tangential velocity from its pose
    # after 15 steps; the hinge is an ALM penalty, so the radial component is
    # only weakly observable and the fit trades a little of one for the other
    sc = pendulum()
    spec = diff.ParamSpec(["velocity"], bodies=[1])
    truth = np.array([0.0, 0.8, 0.0])
    target = diff.rollout(sc, spec, truth, 15, [1], oracle_runner)
    theta, hist = diff.fit(sc, spec, spec.get(sc), target, 15, [1], iters=4, runner=oracle_runner)
    assert hist[0] > 1e-6 and hist[-1] < 1e-12 * hist[0]
    assert abs(theta[1] - truth[1]) <= 1e-4 and abs(theta[0]) <= 1e-2
