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


# ---------------------------------------------------------------------------
# Identification against the reference's double-pendulum trajectory data
# (tests/golden/double_pendulum: nexdynipc/assets/reference_data/
# double_pendulum/Link{1,2}_Pos.csv thinned by make_double_pendulum_reference.py)
# ---------------------------------------------------------------------------
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "double_pendulum")
# the reference's scene file (assets/double_pendulum/double_pendulum.json),
# copied by make_double_pendulum_reference.py
REF_SCENE = os.path.join(GOLDEN, "double_pendulum.json")


def oracle_sampler(worlds, steps, every):
    out = []
    for w in worlds:
        ow = refcpu.OracleWorld(w)
        res, done = [], 0
        for c in diff.sample_counts(steps, every):
            for _ in range(int(c) - done):
                ow.step()
            done = int(c)
            res.append(ow.state())
        out.append(res)
    return out


def pendulum_reference(every=10):
    ref = [diff.load_reference_csv(os.path.join(GOLDEN, f"Link{k}_Pos.csv")) for k in (1, 2)]
    sc = scenes.double_pendulum()
    t = sc.dt * diff.sample_counts(sc.steps, every)
    return ref, t, np.stack([diff.reference_at(t, r) for r in ref], axis=1).reshape(-1)


def test_double_pendulum_builder_is_the_reference_scene():
    import dataclasses
    from nexdynipc_b200 import sceneio
    a = scenes.double_pendulum()
    b, _ = sceneio.load_scene(REF_SCENE)
    for f in dataclasses.fields(a):
        if f.name in ("body_ids", "body_names", "name"):
            continue
        va, vb = getattr(a, f.name), getattr(b, f.name)
        if f.name == "settings":
            assert bytes(va) == bytes(vb)
        elif isinstance(va, np.ndarray) or isinstance(vb, np.ndarray):
            assert np.array_equal(va, vb), f.name
        else:
            assert va == vb, f.name


def test_sample_counts_and_reference_helpers():
    assert list(diff.sample_counts(30, 10)) == [10, 20, 30]
    assert list(diff.sample_counts(25, 10)) == [10, 20, 25]
    with pytest.raises(ValueError):
        diff.sample_counts(0, 10)
    ref = diff.load_reference_csv(os.path.join(GOLDEN, "Link2_Pos.csv"))
    assert ref.shape == (302, 4) and ref[0, 0] == 0.0 and ref[0, 1] == 1.5 and ref[-1, 0] > 1.5
    assert np.all(np.diff(ref[:, 0]) > 0)
    # at the file's own times the interpolant is the data
    assert np.array_equal(diff.reference_at(ref[:5, 0], ref), ref[:5, 1:])
    mid = 0.5 * (ref[3, 0] + ref[4, 0])
    assert np.allclose(diff.reference_at([mid], ref)[0], 0.5 * (ref[3, 1:] + ref[4, 1:]), rtol=0, atol=1e-15)
    P = ref[:, 1:]
    assert diff.rmse_distance(P, P) == 0.0
    assert diff.rmse_distance(P + np.array([0.003, 0.004, 0.0]), P) == pytest.approx(0.005, rel=1e-12)


def test_inertia_parameters_round_trip():
    sc = scenes.double_pendulum(inertia_zz=(0.7, 1.3))
    spec = diff.ParamSpec(["inertia", "mass"], bodies=[1, 2], inertia_axes=[2])
    assert spec.size() == 4
    th = spec.get(sc)
    assert np.array_equal(th, [0.7, 1.3, 1.0, 1.0])
    s2 = spec.put(sc, [0.9, 1.1, 2.0, 3.0])
    assert s2.inertia[1, 8] == 0.9 and s2.inertia[2, 8] == 1.1 and s2.inertia[1, 0] == 1.0
    assert np.array_equal(s2.mass, [1.0, 2.0, 3.0]) and sc.inertia[1, 8] == 0.7
    assert spec.feasible([0.9, 1.1, 2.0, 3.0]) and not spec.feasible([0.9, -1.0, 2.0, 3.0])
    assert not spec.feasible([0.9, np.nan, 2.0, 3.0])
    with pytest.raises(ValueError):
        diff.ParamSpec(["stiffness"]).size()


def test_identify_link_inertias_from_reference_data():
    # the reference data fits the scene file's unit inertias: from a wrong
    # guess, Gauss-Newton on the sampled positions (every 10 ms over 1.5 s)
    # recovers the links' inertia about the hinge axis to 1 %, and the
    # position RMSE against the data drops below 1 mm for both links
    ref, t, target = pendulum_reference()
    sc = scenes.double_pendulum(inertia_zz=(0.6, 1.6))
    spec = diff.ParamSpec(["inertia"], bodies=[1, 2], inertia_axes=[2])
    theta, hist = diff.fit_trajectory(sc, spec, spec.get(sc), target, sc.steps, [1, 2], 10, iters=4,
                                      sampler=oracle_sampler)
    assert np.all(np.abs(theta - 1.0) < 0.01), theta
    assert hist[-1] < 1e-4 * hist[0] and all(b <= a for a, b in zip(hist, hist[1:]))
    y = diff.sampled_positions(oracle_sampler([spec.put(sc, theta)], sc.steps, 10)[0], [1, 2]).reshape(-1, 2, 3)
    for j in range(2):
        assert diff.rmse_distance(y[:, j], diff.reference_at(t, ref[j])) < 1e-3


@pytest.mark.gpu
def test_device_identification_matches_the_oracle():
    # the same identification with the 2P + 1 worlds stepped as one device
    # batch: sampled positions within 1e-6 m of the oracle's, same estimate
    ref, t, target = pendulum_reference()
    sc = scenes.double_pendulum(inertia_zz=(0.6, 1.6))
    spec = diff.ParamSpec(["inertia"], bodies=[1, 2], inertia_axes=[2])
    _, yg, Jg = diff.trajectory_jacobian(sc, spec, spec.get(sc), sc.steps, [1, 2], 10)
    _, yo, Jo = diff.trajectory_jacobian(sc, spec, spec.get(sc), sc.steps, [1, 2], 10, sampler=oracle_sampler)
    assert np.abs(yg - yo).max() <= 1e-6
    # a position difference d moves a central difference by d / h (h = 1e-6)
    assert np.abs(Jg - Jo).max() <= 1e-2 * np.abs(Jo).max()
    theta, hist = diff.fit_trajectory(sc, spec, spec.get(sc), target, sc.steps, [1, 2], 10, iters=4)
    assert np.all(np.abs(theta - 1.0) < 0.01), theta
    assert hist[-1] < 1e-4 * hist[0]


def test_oracle_double_pendulum_follows_the_reference_data():
    # the reference's double-pendulum case with the scene file's parameters:
    # the restated step stays within 1 mm (link 1) and 2 mm (link 2) RMS of
    # the reference's trajectory data over the 1.5 s the file simulates
    ref, t, target = pendulum_reference()
    sc = scenes.double_pendulum()
    y = diff.sampled_positions(oracle_sampler([sc], sc.steps, 10)[0], [1, 2]).reshape(-1, 2, 3)
    e1 = diff.rmse_distance(y[:, 0], diff.reference_at(t, ref[0]))
    e2 = diff.rmse_distance(y[:, 1], diff.reference_at(t, ref[1]))
    assert e1 < 1e-3 and e2 < 2e-3, (e1, e2)
    # the links swing through metres, so the match is not trivial
    assert np.abs(target.reshape(-1, 2, 3)[:, 1] - np.array([1.5, 0.0, 0.0])).max() > 1.0
