"""Control forms of World::forms in the CPU oracle: DampedSpringForm,
PositionDriveForm, LinearVelocityDriveForm and ForceDriveForm
(src/Control/*.cpp), against their closed forms, central differences of their
own values, and the velocity-drive KPI rule of IPCSolver.cpp:1197-1215."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu


def two_boxes(add_form, vel_b=(0.0, 0.0, 0.0)):
    sb = scenes.SceneBuilder("pair")
    v, f = scenes.box_mesh(0.05, 0.05, 0.05)
    sb.add_body(v, f, (0.0, 1.0, 0.0), mass=1.0, inertia=np.eye(3), vel=(0.1, -0.2, 0.05))
    sb.add_body(v, f, (0.3, 0.8, 0.1), mass=1.0, inertia=np.eye(3), vel=vel_b)
    add_form(sb)
    return sb.build(abi.default_settings(), 0.01, 1)


def oracle_at(sc):
    w = refcpu.OracleWorld(sc)
    w.set_form_state(np.zeros(0, dtype=abi.CONTACT_DTYPE), None, np.zeros(12))
    x = np.zeros(12)
    x[0:3], x[6:9] = sc.position[0], sc.position[1]
    x[3:6], x[9:12] = (0.01, -0.02, 0.03), (0.02, 0.01, -0.01)
    return w, x


def fd_gradient(w, x, h=1e-7):
    g = np.zeros_like(x)
    for k in range(len(x)):
        xp, xm = x.copy(), x.copy()
        xp[k] += h
        xm[k] -= h
        g[k] = (w.form_value(abi.NXD_FORM_DRIVES, xp) - w.form_value(abi.NXD_FORM_DRIVES, xm)) / (2 * h)
    return g


def test_damped_spring_value_gradient_hessian():
    # DampedSpringForm.cpp:54-112: E = k/2 (|pB - pA| - L)^2; the gradient
    # adds c (vB - vA).d to the traction; the Hessian is k d d^T per block
    k, L, c = 300.0, 0.2, 4.0
    sc = two_boxes(lambda sb: sb.damped_spring(0, 1, L, k, c), vel_b=(0.3, 0.1, -0.2))
    w, x = oracle_at(sc)
    dv = x[6:9] - x[0:3]
    ln = np.linalg.norm(dv)
    d = dv / ln
    assert w.form_value(abi.NXD_FORM_DRIVES, x) == pytest.approx(0.5 * k * (ln - L) ** 2, rel=1e-14)
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    vrel = (sc.velocity[1] - sc.velocity[0]) @ d
    tr = (k * (ln - L) + c * vrel) * d
    assert np.allclose(g[6:9], tr, rtol=1e-14, atol=0) and np.allclose(g[0:3], -tr, rtol=1e-14, atol=0)
    assert np.all(g[3:6] == 0) and np.all(g[9:12] == 0)
    H = w.form_hessian(abi.NXD_FORM_DRIVES, x)
    K = k * np.outer(d, d)
    assert np.allclose(H[0:3, 0:3], K, rtol=1e-14, atol=1e-12) and np.allclose(H[6:9, 6:9], K, rtol=1e-14, atol=1e-12)
    assert np.allclose(H[0:3, 6:9], -K, rtol=1e-14, atol=1e-12) and np.allclose(H[6:9, 0:3], -K, rtol=1e-14, atol=1e-12)
    # without damping the gradient is the derivative of the value
    sc0 = two_boxes(lambda sb: sb.damped_spring(0, 1, L, k, 0.0), vel_b=(0.3, 0.1, -0.2))
    w0, x0 = oracle_at(sc0)
    assert np.allclose(w0.form_gradient(abi.NXD_FORM_DRIVES, x0), fd_gradient(w0, x0), rtol=0, atol=1e-5)


def test_damped_spring_degenerate_direction_is_unit_x():
    sc = two_boxes(lambda sb: sb.damped_spring(0, 1, 0.1, 50.0, 0.0))
    w, x = oracle_at(sc)
    x[6:9] = x[0:3]
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    assert g[6] == pytest.approx(50.0 * (0.0 - 0.1)) and g[7] == 0 and g[8] == 0


@pytest.mark.parametrize("max_force,deadzone", [(0.0, 0.0), (3.0, 0.0), (3.0, 0.02), (0.0, 0.05)])
def test_position_drive(max_force, deadzone):
    # PositionDriveForm.cpp:66-170: e = dz(target - (pB - pA).a), force k e or
    # m tanh(k e / m); the gradient is minus the force along the axis on B
    kp, tgt = 40.0, 0.1
    axis = np.array([1.0, 0.5, -0.2])
    sc = two_boxes(lambda sb: sb.position_drive(0, 1, axis, kp, tgt, max_force=max_force, deadzone=deadzone))
    w, x = oracle_at(sc)
    a = axis / np.linalg.norm(axis)
    err = tgt - (x[6:9] - x[0:3]) @ a
    e = err if deadzone <= 0 else (err - deadzone if err > deadzone else (err + deadzone if err < -deadzone else 0.0))
    force = kp * e if max_force <= 0 else max_force * np.tanh(kp * e / max_force)
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    assert np.allclose(g[6:9], -force * a, rtol=1e-13, atol=1e-14)
    assert np.allclose(g[0:3], force * a, rtol=1e-13, atol=1e-14)
    assert np.allclose(g, fd_gradient(w, x), rtol=0, atol=1e-5)
    H = w.form_hessian(abi.NXD_FORM_DRIVES, x)
    h = kp if max_force <= 0 else (0.0 if abs(err) <= deadzone else kp * (1 - np.tanh(kp * e / max_force) ** 2))
    assert np.allclose(H[6:9, 6:9], h * np.outer(a, a), rtol=1e-13, atol=1e-13)
    assert np.allclose(H[0:3, 6:9], -h * np.outer(a, a), rtol=1e-13, atol=1e-13)


def test_position_drive_to_world():
    sc = two_boxes(lambda sb: sb.position_drive(-1, 1, (0, 1, 0), 10.0, 0.5))
    w, x = oracle_at(sc)
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    assert g[7] == pytest.approx(-10.0 * (0.5 - x[7]), rel=1e-14)
    assert np.all(g[0:6] == 0)


def test_force_drive_gradient_and_value():
    # ForceDriveForm.cpp:22-40: zero energy, gradient minus the force / torque
    F, T = np.array([1.0, -2.0, 0.5]), np.array([0.1, 0.0, -0.3])
    sc = two_boxes(lambda sb: sb.force_drive(1, F, T))
    w, x = oracle_at(sc)
    assert w.form_value(abi.NXD_FORM_DRIVES, x) == 0.0
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    assert np.array_equal(g[6:9], -F) and np.array_equal(g[9:12], -T) and np.all(g[0:6] == 0)
    assert np.all(w.form_hessian(abi.NXD_FORM_DRIVES, x) == 0)


def test_linear_velocity_drive_first_call_and_state():
    # LinearVelocityDriveForm.cpp:113-219: the first call after the step's
    # set-up sees zero joint velocity; later calls difference against the
    # previous call's positions
    kv, vt, dt = 2.0, 0.7, 0.01
    sc = two_boxes(lambda sb: sb.linear_velocity_drive(0, 1, (0, 0, 2.0), kv, vt))
    w, x = oracle_at(sc)
    g = w.form_gradient(abi.NXD_FORM_DRIVES, x)
    assert g[8] == pytest.approx(-(kv * vt) / dt, rel=1e-14) and g[2] == pytest.approx((kv * vt) / dt, rel=1e-14)
    x2 = x.copy()
    x2[8] += 0.003                        # B moved 3 mm along the axis: 0.3 m/s
    g2 = w.form_gradient(abi.NXD_FORM_DRIVES, x2)
    assert g2[8] == pytest.approx(-(kv * (vt - 0.3)) / dt, rel=1e-12)
    H = w.form_hessian(abi.NXD_FORM_DRIVES, x2)
    assert H[8, 8] == pytest.approx(kv / dt ** 2, rel=1e-14) and H[2, 8] == pytest.approx(-kv / dt ** 2, rel=1e-14)


def test_kpi_counts_only_angular_velocity_drives():
    sc = scenes.control_forms()
    ow = refcpu.OracleWorld(sc)
    for _ in range(35):
        ow.step()
    d = ow.diagnostics()
    # the one VelocityDriveForm saturates; the five other control forms are
    # not counted, so the ratio is 1 (not 1/6)
    assert d["last_torque_saturation_ratio"] == 1.0
    assert d["last_angular_velocity_error"] > 0.0


def test_control_forms_scene_runs_in_the_oracle():
    sc = scenes.control_forms()
    ow = refcpu.OracleWorld(sc)
    y0 = sc.position[6, 1]
    for _ in range(30):
        ow.step()
    st = ow.state()
    assert np.isfinite(st["position"]).all()
    # the force drive's 4 N upward on a 1 kg box: it falls slower than free fall
    free = y0 + sc.velocity[6, 1] * 0.3 - 0.5 * 9.81 * 0.3 ** 2
    assert st["position"][6, 1] > free
    assert ow.diagnostics()["status"] == 0


def test_invalid_control_forms_are_refused():
    for bad in (lambda sb: sb.damped_spring(-1, 1, 0.1, 1.0, 0.0),
                lambda sb: sb.damped_spring(1, 1, 0.1, 1.0, 0.0),
                lambda sb: sb.force_drive(7, (1, 0, 0))):
        sc = two_boxes(bad)
        with pytest.raises(RuntimeError):
            refcpu.OracleWorld(sc)
