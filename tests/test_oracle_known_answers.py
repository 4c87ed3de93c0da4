"""The CPU oracle against the known answers of the reference's own tests.

Each case restates an assertion of NexDynIPC's Catch2 suite (file:line in the
test names) and runs it against oracle/refcpu, pinning the restatement where
the reference's tests pin behaviour.
"""
import math

import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu


def L():
    return refcpu.lib()


def fval(u, N, mu, eps=1e-8):
    return L().nxo_friction_value(refcpu._d(u), N, mu, eps)


def fgrad(u, N, mu, eps=1e-8):
    g = np.zeros(3)
    L().nxo_friction_gradient(refcpu._d(u), N, mu, eps, abi.dptr(g))
    return g


def fhess(u, N, mu, eps=1e-8):
    H = np.zeros(9)
    L().nxo_friction_hessian(refcpu._d(u), N, mu, eps, abi.dptr(H))
    return H.reshape(3, 3)


# tests/physics/test_friction.cpp:15-84
def test_friction_potential_basic():
    u = np.array([0.1, 0, 0])
    assert fval(u, 10.0, 0.5) > 0
    assert fval(u, 0.0, 0.5) == 0.0
    assert fval(np.array([0.2, 0, 0]), 10.0, 0.5) > fval(u, 10.0, 0.5)
    g = fgrad(u, 10.0, 0.5)
    assert g[0] > 0 and abs(g[1]) < 1e-10 and abs(g[2]) < 1e-10
    H = fhess(np.array([0.1, 0.05, 0]), 10.0, 0.5)
    assert np.abs(H - H.T).max() < 1e-10
    assert np.linalg.eigvalsh(H).min() >= -1e-10


# tests/physics/test_friction.cpp:86-127
def test_friction_smooth_exact_values():
    N, mu, eps = 10.0, 0.5, 0.1
    u = np.array([0.05, 0, 0])
    v = L().nxo_friction_value_smooth(refcpu._d(u), N, mu, eps)
    assert abs(v - 0.5 * mu * N / eps * float(u @ u)) < 1e-10
    u = np.array([0.5, 0, 0])
    v = L().nxo_friction_value_smooth(refcpu._d(u), N, mu, eps)
    assert abs(v - mu * N * (np.linalg.norm(u) - 0.5 * eps)) < 1e-10
    assert L().nxo_friction_value_smooth(refcpu._d(np.array([0.1, 0, 0])), N, mu, 1e-8) > 0


# tests/physics/test_friction.cpp:299-326 and 388-416
def test_friction_fd_gradient_and_hessian():
    u = np.array([0.1, 0.05, 0.02])
    N, mu, eps, h = 10.0, 0.5, 1e-8, 1e-6
    g = fgrad(u, N, mu, eps)
    H = fhess(u, N, mu, eps)
    for i in range(3):
        e = np.zeros(3); e[i] = h
        fd = (fval(u + e, N, mu, eps) - fval(u - e, N, mu, eps)) / (2 * h)
        assert abs(g[i] - fd) < 1e-5
        fdh = (fgrad(u + e, N, mu, eps) - fgrad(u - e, N, mu, eps)) / (2 * h)
        for r in range(3):
            assert abs(H[r, i] - fdh[r]) < 1e-4


# src/Physics/Contact/Barrier.cpp semantics, tests/physics/test_ccd.cpp:163-210
def test_barrier_shape():
    dh, k = 1e-3, 1e4
    assert L().nxo_barrier_value(2e-3, dh, k) == 0.0
    assert L().nxo_barrier_value(0.0, dh, k) == math.inf
    assert L().nxo_barrier_value(5e-4, dh, k) > 0
    assert L().nxo_barrier_gradient(5e-4, dh, k) < 0
    assert L().nxo_barrier_hessian(5e-4, dh, k) > 0
    d = 4e-4
    v = -k * (d - dh) ** 2 * math.log(d / dh)
    assert abs(L().nxo_barrier_value(d, dh, k) - v) <= 1e-15 * abs(v)
    h = 1e-9
    fd = (L().nxo_barrier_value(d + h, dh, k) - L().nxo_barrier_value(d - h, dh, k)) / (2 * h)
    assert abs(L().nxo_barrier_gradient(d, dh, k) - fd) < 1e-5 * abs(fd)


def root_poly(coeffs, lo=0.0, hi=1.0, tol=1e-8):
    c = np.asarray(coeffs, dtype=np.float64)
    rl, rh = np.zeros(1), np.zeros(1)
    found = L().nxo_interval_root_poly(abi.dptr(c), len(c) - 1, lo, hi, tol, abi.dptr(rl), abi.dptr(rh))
    return found, rl[0], rh[0]


# tests/physics/test_ccd.cpp:79-125
def test_interval_root_finder():
    f, lo, hi = root_poly([-0.5, 1.0])
    assert f and abs(lo - 0.5) < 1e-6 and abs(hi - 0.5) < 1e-6
    f, lo, hi = root_poly([-0.25, 0.0, 1.0])
    assert f and abs(lo - 0.5) < 1e-6
    f, _, _ = root_poly([1.0, 0.0, 1.0])
    assert not f


def two_body_scene(q0=(1, 0, 0, 0), q1=(1, 0, 0, 0), p1=(1, 0, 0)):
    sb = scenes.SceneBuilder("two")
    v, f = scenes.box_mesh(0.1, 0.1, 0.1)
    sb.add_body(v, f, (0, 0, 0), quat=q0, mass=1.0, inertia=np.eye(3))
    sb.add_body(v, f, p1, quat=q1, mass=1.0, inertia=np.eye(3))
    s = abi.default_settings()
    s.enable_friction = 1
    s.friction_coeff = 0.5
    return sb.build(s, 0.01, 1)


def contact(a, b, point, normal, dist=0.0):
    c = np.zeros(1, dtype=abi.CONTACT_DTYPE)
    c["body_a"], c["body_b"] = a, b
    c["point"][0] = point
    c["normal"][0] = normal
    c["distance"] = dist
    return c


# tests/physics/test_friction.cpp:222-297
def test_friction_form_tangent_displacement_follows_iterate():
    sc = two_body_scene()
    sc.velocity[0] = (100.0, 0, 0)
    w = refcpu.OracleWorld(sc)
    w.set_form_state(contact(0, 1, (0, 0, 0), (0, 1, 0)), normal_forces=[5.0], x_hat=np.zeros(12), dt=0.01)
    x = np.zeros(12)
    x[6:9] = (1, 0, 0)
    assert abs(w.form_value(abi.NXD_FORM_FRICTION, x)) < 1e-12
    x[0] = 0.02
    assert w.form_value(abi.NXD_FORM_FRICTION, x) > 0.0


# tests/physics/test_friction.cpp:328-386 (rotational FD, tolerance 6e-2)
def test_friction_form_rotational_fd():
    qa = scenes.quat_from_axis_angle((0, 1, 0), 0.4)
    qb = scenes.quat_from_axis_angle((1, 0, 0), -0.2)
    sc = two_body_scene(qa, qb)
    w = refcpu.OracleWorld(sc)
    w.set_form_state(contact(0, 1, (0, 0, 1), (0, 1, 0)), normal_forces=[5.0], x_hat=np.zeros(12), dt=0.01)
    x = np.zeros(12)
    x[6:9] = (1, 0, 0)
    x[4] = 0.005
    x[10] = -0.003
    g = w.form_gradient(abi.NXD_FORM_FRICTION, x)
    h = 1e-6
    for idx in (4, 10):
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        fd = (w.form_value(abi.NXD_FORM_FRICTION, xp) - w.form_value(abi.NXD_FORM_FRICTION, xm)) / (2 * h)
        # the reference runs this case with eps 1e-4; with the step's eps
        # 1e-8 the potential is |u| to within 1e-8, so the same bound holds
        assert abs(g[idx] - fd) < 6e-2


def fixed_scene(pos, target, quat=(1, 0, 0, 0)):
    sb = scenes.SceneBuilder("fixed")
    v, f = scenes.box_mesh(0.1, 0.1, 0.1)
    sb.add_body(v, f, pos, quat=quat, mass=1.0, inertia=np.eye(3))
    p = np.zeros(16)
    p[0:3] = target
    p[3:7] = (1, 0, 0, 0)
    sb.joints.append((abi.NXD_JOINT_FIXED, 0, -1, p, 1e8))
    return sb.build(abi.default_settings(), 0.01, 1)


# tests/dynamics/test_joint.cpp:86-140
def test_fixed_joint_known_values():
    sc = fixed_scene((1, 2, 3), (1, 2, 3))
    w = refcpu.OracleWorld(sc)
    w.set_form_state(np.zeros(0, dtype=abi.CONTACT_DTYPE), None, np.zeros(6))
    x = np.array([1, 2, 3, 0, 0, 0.0])
    assert abs(w.form_value(abi.NXD_FORM_CONSTRAINT, x)) < 1e-10
    sc = fixed_scene((2, 3, 4), (1, 2, 3))
    w = refcpu.OracleWorld(sc)
    w.set_form_state(np.zeros(0, dtype=abi.CONTACT_DTYPE), None, np.zeros(6))
    x = np.array([2, 3, 4, 0, 0, 0.0])
    # C = (1,1,1,0,0,0), E = 0.5 mu |C|^2, grad = J^T mu C
    assert abs(w.form_value(abi.NXD_FORM_CONSTRAINT, x) - 0.5 * 1e8 * 3) < 1e-6
    g = w.form_gradient(abi.NXD_FORM_CONSTRAINT, x)
    assert np.allclose(g, [1e8, 1e8, 1e8, 0, 0, 0])
    H = w.form_hessian(abi.NXD_FORM_CONSTRAINT, x)
    assert np.allclose(H, 1e8 * np.eye(6))


def hinge_scene(pa, pb, qa=(1, 0, 0, 0), qb=(1, 0, 0, 0), axis_b=(0, 0, 1)):
    sb = scenes.SceneBuilder("hinge")
    v, f = scenes.box_mesh(0.1, 0.1, 0.1)
    sb.add_body(v, f, pa, quat=qa, mass=1.0, inertia=np.eye(3))
    sb.add_body(v, f, pb, quat=qb, mass=1.0, inertia=np.eye(3))
    sb.hinge(0, 1, (0, 0, 0), (0, 0, 0), (0, 0, 1), axis_b)
    return sb.build(abi.default_settings(), 0.01, 1)


# tests/dynamics/test_joint.cpp:185-260 (hinge), 600-655 (Jacobian by FD)
def test_hinge_joint_constraint_and_fd_gradient():
    sc = hinge_scene((0, 0, 0), (0, 0, 0))
    w = refcpu.OracleWorld(sc)
    w.set_form_state(np.zeros(0, dtype=abi.CONTACT_DTYPE), None, np.zeros(12))
    x = np.zeros(12)
    assert abs(w.form_value(abi.NXD_FORM_CONSTRAINT, x)) < 1e-20
    x = np.array([0.01, -0.02, 0.03, 0.001, 0.002, -0.003, -0.01, 0.02, 0.0, 0.0, 0.004, 0.001])
    g = w.form_gradient(abi.NXD_FORM_CONSTRAINT, x)
    # the reference's Jacobian is the left-perturbation one (exact at
    # theta = 0, first order in |theta| elsewhere), so compare with FD
    # relative to the gradient's scale
    h = 1e-7
    gmax = np.abs(g).max()
    for k in range(12):
        xp, xm = x.copy(), x.copy()
        xp[k] += h
        xm[k] -= h
        fd = (w.form_value(abi.NXD_FORM_CONSTRAINT, xp) - w.form_value(abi.NXD_FORM_CONSTRAINT, xm)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-3 * gmax


# tests/physics/test_contact_regression.cpp:98-123: separated bodies give no pairs,
# overlapping boxes give exactly one pair
def test_broad_phase_pairs_known():
    sc = two_body_scene(p1=(0.15, 0, 0))
    w = refcpu.OracleWorld(sc)
    assert w.body_pairs(0.0).tolist() == [[0, 1]]
    sc = two_body_scene(p1=(5.0, 0, 0))
    w = refcpu.OracleWorld(sc)
    assert len(w.body_pairs(1e-3)) == 0
    # touching boxes intersect (closed intervals, tests/geometry/test_aabb.cpp:136-140)
    sc = two_body_scene(p1=(0.2, 0, 0))
    w = refcpu.OracleWorld(sc)
    assert w.body_pairs(0.0).tolist() == [[0, 1]]


def test_broad_phase_order_descending_j():
    sb = scenes.SceneBuilder("row")
    v, f = scenes.box_mesh(0.1, 0.1, 0.1)
    for i in range(6):
        sb.add_body(v, f, (0.15 * i, 0, 0), mass=1.0, inertia=np.eye(3))
    sc = sb.build(abi.default_settings(), 0.01, 1)
    w = refcpu.OracleWorld(sc)
    p = w.body_pairs(0.2)
    # for each i the reference's BVH traversal reports j in descending order
    for i in range(6):
        js = [b for a, b in p if a == i]
        assert js == sorted(js, reverse=True)
    # gap 0.15|i-j| - 0.2 <= 2 r = 0.4  <=>  |i-j| <= 4
    assert len(p) == 14


# tests/physics/test_ccd.cpp:230-256: CCDSystem returns 1.0 (step dt) without
# face-vertex candidates; the FV root box also never survives the domain test
def test_max_step_is_dt():
    sc = scenes.cube_stack()
    w = refcpu.OracleWorld(sc)
    assert w.max_step(0.01) == 0.01
    sc = two_body_scene(p1=(5.0, 0, 0))
    w = refcpu.OracleWorld(sc)
    assert w.max_step(0.01) == 0.01


def test_literal_and_pruned_min_distance_agree_below_band():
    sc = scenes.cube_stack()
    w = refcpu.OracleWorld(sc)
    lit = w.scene_min_distance(True)
    pr = w.scene_min_distance(False)
    assert lit == pr or (lit >= 1e-6 and pr >= 1e-6)
    # a vertex planted exactly on a face of the body above it
    sb = scenes.SceneBuilder("touch")
    v, f = scenes.box_mesh(0.5, 0.5, 0.5)
    sb.add_body(v, f, (0, 0.0, 0), mass=1.0, inertia=np.eye(3))
    sb.add_body(v, f, (0.3, 1.0, 0.2), mass=1.0, inertia=np.eye(3))
    sc = sb.build(abi.default_settings(), 0.01, 1)
    w = refcpu.OracleWorld(sc)
    lit = w.scene_min_distance(True)
    pr = w.scene_min_distance(False)
    assert lit == pr
    assert lit < 1e-9


def test_newmark_free_fall_recurrence():
    # ImplicitNewmark (TimeIntegration/ImplicitNewmark.cpp): for a free body
    # the Newton solve gives x' = x_tilde + beta h^2 g, so a' = g and
    # v' = v + h ((1 - gamma) a + gamma a'), with a_0 = 0 as the scene starts.
    from nexdynipc_b200 import abi, scenes
    sb = scenes.SceneBuilder("free_fall")
    sb.add_body(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (0.0, 2.0, 0.0), mass=2.0, inertia=np.eye(3),
                vel=(0.3, 1.0, 0.0))
    s = abi.default_settings()
    s.integrator = abi.INTEGRATOR_IMPLICIT_NEWMARK
    s.newmark_beta, s.newmark_gamma = 0.25, 0.5
    h = 0.01
    sc = sb.build(s, h, 50)
    ow = refcpu.OracleWorld(sc)
    g = np.array([0.0, -9.81, 0.0])
    p, v, a = np.array([0.0, 2.0, 0.0]), np.array([0.3, 1.0, 0.0]), np.zeros(3)
    for _ in range(50):
        ow.step()
        xt = p + h * v + h * h * (0.5 - 0.25) * a
        p_new = xt + 0.25 * h * h * g
        a_new = (p_new - xt) / (0.25 * h * h)
        v = v + h * (0.5 * a + 0.5 * a_new)
        p, a = p_new, a_new
    st = ow.state()
    assert np.allclose(st["position"][0], p, rtol=0, atol=1e-10)
    assert np.allclose(st["velocity"][0], v, rtol=0, atol=1e-8)
    assert np.allclose(st["linear_acceleration"][0], g, rtol=0, atol=1e-5)


def slider_scene(kind):
    """Two boxes joined by a prismatic / cylindrical joint, or kept within a
    distance band (PrismaticJoint, CylindricalJoint, DistanceLimitJoint)."""
    sb = scenes.SceneBuilder(kind)
    v, f = scenes.box_mesh(0.1, 0.1, 0.1)
    sb.add_body(v, f, (0, 0, 0), mass=1.0, inertia=np.eye(3))
    sb.add_body(v, f, (0.3, 0.1, 0), quat=scenes.quat_from_axis_angle((0, 0, 1), 0.2), mass=1.0, inertia=np.eye(3))
    if kind == "prismatic":
        sb.prismatic(0, 1, (0.1, 0, 0), (-0.1, 0, 0), (1, 0.2, 0), (1, 0, 0.1), stiffness=1e4)
    elif kind == "cylindrical":
        sb.cylindrical(0, 1, (0.1, 0, 0), (-0.1, 0, 0), (0.3, 1, 0), (0, 1, 0), stiffness=1e4)
    else:
        sb.distance_limit(0, 1, 0.4, 0.5, stiffness=1e4)
    return sb.build(abi.default_settings(), 0.01, 1)


@pytest.mark.parametrize("kind", ["prismatic", "cylindrical", "distance"])
def test_new_joints_constraint_fd_gradient(kind):
    # PrismaticJoint / CylindricalJoint / DistanceLimitJoint: the constraint
    # form's gradient J^T (mu C + lambda) against central differences of its
    # value (the rotational columns are the left-perturbation Jacobian,
    # exact at theta = 0)
    sc = slider_scene(kind)
    w = refcpu.OracleWorld(sc)
    w.set_form_state(np.zeros(0, dtype=abi.CONTACT_DTYPE), None, np.zeros(12))
    x = np.zeros(12)
    x[0:3] = sc.position[0]
    x[6:9] = sc.position[1] + (0.0, 0.0, 0.0 if kind != "distance" else 0.5)   # distance 0.59 > max 0.5
    e0 = w.form_value(abi.NXD_FORM_CONSTRAINT, x)
    assert e0 > 0.0
    g = w.form_gradient(abi.NXD_FORM_CONSTRAINT, x)
    h = 1e-7
    for k in range(12):
        xp, xm = x.copy(), x.copy()
        xp[k] += h
        xm[k] -= h
        fd = (w.form_value(abi.NXD_FORM_CONSTRAINT, xp) - w.form_value(abi.NXD_FORM_CONSTRAINT, xm)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-5 * np.abs(g).max(), (kind, k, g[k], fd)
    H = w.form_hessian(abi.NXD_FORM_CONSTRAINT, x)
    assert np.allclose(H, H.T, rtol=0, atol=1e-9 * np.abs(H).max())
    assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()
