"""GPU parity: the sm_100a contact step against the CPU oracle on the same
seeded inputs, through the C ABI.

Integer / index outputs (body pairs, candidate lists, contact primitive ids)
must be identical, in the reference's order.  Floating-point outputs are
compared within the parity tolerances: form energies and gradients within
1e-10 relative, trajectories within 1e-6 m / 1e-6 rad; both sides round the
same way (no FMA contraction, same reduction trees), so most of them agree
bit for bit, which the tests report.
"""
import math

import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu

pytestmark = pytest.mark.gpu


def runtime():
    from nexdynipc_b200 import runtime as rt
    return rt


def rows_sorted(a):
    return a[np.lexsort(a.T[::-1])] if len(a) else a


SCENES = {
    "cube_stack": lambda: scenes.cube_stack(),
    "sphere_bowl": lambda: scenes.sphere_bowl(n_spheres=24),
    "hopper_small": lambda: scenes.hopper_chains(n_hulls=192, n_chains=6),
    "control_forms": lambda: scenes.control_forms(),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_body_pairs_and_candidates_identical(name):
    sc = SCENES[name]()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    dh = sc.settings.dhat
    for r in (0.0, dh, 2 * dh, 0.05):
        pg, po = ctx.body_pairs(r), ow.body_pairs(r)
        assert np.array_equal(pg, po), f"pairs differ at r={r}"
    cg, co = ctx.candidates(dh), ow.candidates(dh)
    for k in ("vv", "ev", "ee", "fv"):
        assert len(cg[k]) == len(co[k]), k
        assert np.array_equal(rows_sorted(cg[k]), rows_sorted(co[k])), f"{k} sets differ"
        assert np.array_equal(cg[k], co[k]), f"{k} order differs"


def test_candidates_full_hopper_identical():
    # 1024 hulls + 32 chains: ~10.6k body pairs and ~60M candidates; every
    # hull sits inside the hopper's box, so its 64 vertex scores tie at 0 and
    # the top-32 subset is decided by libstdc++'s introselect data movement.
    sc = scenes.hopper_chains()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    dh = sc.settings.dhat
    cg, co = ctx.candidates(dh), ow.candidates(dh)
    for k in ("vv", "ee", "fv"):
        assert np.array_equal(cg[k], co[k]), k


def contacts_equal(a, b):
    assert len(a) == len(b)
    for f in ("body_a", "body_b", "primitive_type", "primitive_a", "primitive_b"):
        assert np.array_equal(a[f], b[f]), f
    for f in ("point", "normal", "distance"):
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("name", list(SCENES))
def test_contacts_identical(name):
    sc = SCENES[name]()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    cg = ctx.detect_contacts()
    co, _ = ow.detect_contacts()
    contacts_equal(cg, co)
    # detectContactsAtState at a perturbed state (translations and rotations)
    rng = np.random.default_rng(11)
    x = np.zeros(sc.n_bodies * 6)
    for i in range(sc.n_bodies):
        x[6 * i:6 * i + 3] = sc.position[i] + rng.normal(0, 2e-3, 3)
        x[6 * i + 3:6 * i + 6] = rng.normal(0, 2e-3, 3)
    cg = ctx.detect_contacts(x)
    co, _ = ow.detect_contacts(x)
    contacts_equal(cg, co)


def test_contact_cap_and_vv_fallback():
    # a dense pile: more than 2000 raw contacts exercises the distance sort
    sb = scenes.SceneBuilder("pile")
    v, f = scenes.icosphere(2)
    rng = np.random.default_rng(5)
    for i in range(40):
        sb.add_body(v * 0.1, f, rng.uniform(-0.08, 0.08, 3), quat=scenes.random_quaternion(rng))
    s = abi.default_settings()
    s.dhat = 2e-2
    sc = sb.build(s, 0.01, 1)
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    cg = ctx.detect_contacts()
    co, raw = ow.detect_contacts()
    assert raw > 2000 and len(co) == 2000
    # the 2000 kept contacts in libstdc++ std::sort's order (its permutation
    # of equal distances included)
    contacts_equal(cg, co)
    # two far-apart bodies: no pairs, no contacts (empty inputs)
    sb = scenes.SceneBuilder("far")
    bv, bf = scenes.box_mesh(0.1, 0.1, 0.1)
    sb.add_body(bv, bf, (0, 0, 0))
    sb.add_body(bv, bf, (5, 0, 0))
    sc = sb.build(abi.default_settings(), 0.01, 1)
    ctx = runtime().Context(sc)
    assert len(ctx.body_pairs(1e-3)) == 0
    assert len(ctx.detect_contacts()) == 0


def test_scene_min_distance_exact():
    for sc in (scenes.cube_stack(), scenes.sphere_bowl(n_spheres=24)):
        ctx = runtime().Context(sc)
        ow = refcpu.OracleWorld(sc)
        g, c = ctx.scene_min_distance(), ow.scene_min_distance(False)
        assert g == c or (g >= 1e-6 and c >= 1e-6)
    sb = scenes.SceneBuilder("touch")
    v, f = scenes.box_mesh(0.5, 0.5, 0.5)
    sb.add_body(v, f, (0, 0.0, 0), mass=1.0, inertia=np.eye(3))
    sb.add_body(v, f, (0.3, 1.0, 0.2), mass=1.0, inertia=np.eye(3))
    sc = sb.build(abi.default_settings(), 0.01, 1)
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    assert ctx.scene_min_distance() == ow.scene_min_distance(True)


def random_state_and_contacts(sc, seed=3):
    ow = refcpu.OracleWorld(sc)
    rng = np.random.default_rng(seed)
    n = sc.n_bodies
    x = np.zeros(6 * n)
    for i in range(n):
        x[6 * i:6 * i + 3] = sc.position[i] + rng.normal(0, 1e-3, 3)
        x[6 * i + 3:6 * i + 6] = rng.normal(0, 1e-3, 3)
    xh = x + rng.normal(0, 1e-4, 6 * n)
    c, _ = ow.detect_contacts()
    # make part of the barrier active: COM-projected distances below dhat
    nf = np.abs(rng.normal(0, 10.0, len(c))) * (rng.random(len(c)) < 0.7)
    return x, xh, c, nf


@pytest.mark.parametrize("name", ["cube_stack", "hopper_small", "control_forms"])
def test_form_values_gradients_hessian(name):
    sc = SCENES[name]()
    x, xh, c, nf = random_state_and_contacts(sc)
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    ctx.set_form_state(c, nf, xh, sc.dt)
    ow.set_form_state(c, nf, xh, sc.dt)
    for form in range(8):
        vg = ctx.form_value(form, x)
        vo = ow.form_value(form, x)
        assert abs(vg - vo) <= 1e-10 * max(1.0, abs(vo)), (form, vg, vo)
        gg = ctx.form_gradient(form, x)
        go = ow.form_gradient(form, x)
        assert np.abs(gg - go).max() <= 1e-10 * max(1.0, np.abs(go).max()), form
    Hg = ctx.form_hessian_dense(x)
    Ho = ow.form_hessian(abi.NXD_FORM_TOTAL, x)
    assert np.abs(Hg - Ho).max() <= 1e-10 * max(1.0, np.abs(Ho).max())
    ng = ctx.normal_forces(x, len(c))
    no = ow.normal_forces(x, len(c))
    assert np.array_equal(ng, no)


def quat_angle(qa, qb):
    d = np.abs(np.einsum("ij,ij->i", qa, qb)).clip(0, 1)
    return 2 * np.arccos(d)


def run_pair(sc, steps, check_every=1):
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    worst_p = worst_r = 0.0
    for k in range(steps):
        ctx.step()
        ow.step()
        if (k + 1) % check_every and k + 1 != steps:
            continue
        sg, so = ctx.state(), ow.state()
        worst_p = max(worst_p, float(np.abs(sg["position"] - so["position"]).max()))
        worst_r = max(worst_r, float(quat_angle(sg["orientation"], so["orientation"]).max()))
        dg, do = ctx.diagnostics(), ow.diagnostics()
        assert dg["kappa"] == do["kappa"]
        assert dg["n_contacts"] == do["n_contacts"]
        assert dg["alm_iterations"] == do["alm_iterations"]
        assert dg["status"] == 0
    lg, mg = ctx.joint_state()
    lo, mo = ow.joint_state()
    return worst_p, worst_r, (lg, mg, lo, mo)


def test_trajectory_cube_stack_100_steps():
    wp, wr, (lg, mg, lo, mo) = run_pair(scenes.cube_stack(), 100)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)
    assert np.array_equal(mg, mo)


def test_trajectory_sphere_bowl():
    wp, wr, _ = run_pair(scenes.sphere_bowl(n_spheres=32), 30, check_every=5)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)


def test_trajectory_hopper_chains_small():
    wp, wr, (lg, mg, lo, mo) = run_pair(scenes.hopper_chains(n_hulls=128, n_chains=8), 20, check_every=5)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)
    assert np.allclose(mg, mo, rtol=0, atol=0)
    assert np.abs(lg - lo).max() <= 1e-6 * max(1.0, np.abs(lo).max())


def double_pendulum():
    # the reference's built-in double pendulum (src/App/SceneLoader.cpp:567-621):
    # bodies without meshes, one fixed anchor and two hinged links
    sb = scenes.SceneBuilder("double_pendulum")
    empty_v = np.zeros((0, 3))
    empty_f = np.zeros((0, 3), np.int32)
    sb.add_body(empty_v, empty_f, (0, 0, 0), mass=1.0, inertia=np.eye(3))
    sb.fix(0)
    sb.add_body(empty_v, empty_f, (0.5, 0, 0), mass=1.0, inertia=np.eye(3))
    sb.add_body(empty_v, empty_f, (1.5, 0, 0), mass=1.0, inertia=np.eye(3))
    sb.hinge(0, 1, (0, 0, 0), (-0.5, 0, 0), (0, 0, 1), (0, 0, 1))
    sb.hinge(1, 2, (0.5, 0, 0), (-0.5, 0, 0), (0, 0, 1), (0, 0, 1))
    s = abi.default_settings()
    s.alm_max_iters = 6
    return sb.build(s, 0.01, 100)


def test_trajectory_double_pendulum_meshless():
    wp, wr, _ = run_pair(double_pendulum(), 100, check_every=10)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)


def test_trajectory_newmark():
    # the reference's Simulation default integrator (ImplicitNewmark, beta
    # 0.25, gamma 0.5) on the double pendulum and the cube stack
    for sc, steps in ((double_pendulum(), 100), (scenes.cube_stack(), 50)):
        sc.settings.integrator = abi.INTEGRATOR_IMPLICIT_NEWMARK
        wp, wr, _ = run_pair(sc, steps, check_every=10)
        assert wp <= 1e-6 and wr <= 1e-6, (sc.name, wp, wr)


def test_trajectory_prismatic_cylindrical_distance_joints():
    # PrismaticJoint, CylindricalJoint and DistanceLimitJoint on falling
    # bodies hanging from a fixed anchor (ALM terms, hardening, active sets)
    sb = scenes.SceneBuilder("sliders")
    v, f = scenes.box_mesh(0.05, 0.05, 0.05)
    a = sb.add_body(v, f, (0.0, 1.0, 0.0), mass=1.0, inertia=0.01 * np.eye(3))
    sb.fix(a)
    b = sb.add_body(v, f, (0.2, 1.0, 0.0), mass=0.5, inertia=0.01 * np.eye(3), vel=(0.1, 0.0, 0.2))
    c = sb.add_body(v, f, (0.2, 0.7, 0.0), mass=0.5, inertia=0.01 * np.eye(3), omega=(0.0, 1.0, 0.0))
    d = sb.add_body(v, f, (0.5, 0.7, 0.1), mass=0.5, inertia=0.01 * np.eye(3), vel=(0.0, 0.3, 0.0))
    sb.prismatic(a, b, (0.1, 0, 0), (-0.1, 0, 0), (1, 0, 0), (1, 0, 0), stiffness=1e6)
    sb.cylindrical(b, c, (0, -0.15, 0), (0, 0.15, 0), (0, 1, 0), (0, 1, 0), stiffness=1e6)
    sb.distance_limit(c, d, 0.2, 0.32, stiffness=1e6)
    s = abi.default_settings()
    s.alm_max_iters = 6
    sc = sb.build(s, 0.01, 60)
    wp, wr, (lg, mg, lo, mo) = run_pair(sc, 60, check_every=10)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)
    assert np.abs(lg - lo).max() <= 1e-6 * max(1.0, np.abs(lo).max())


def test_trajectory_control_forms():
    # DampedSpringForm, PositionDriveForm (to the world and between bodies),
    # LinearVelocityDriveForm, VelocityDriveForm and ForceDriveForm in one
    # World::forms list, with contacts on a ground box
    wp, wr, _ = run_pair(scenes.control_forms(), 60, check_every=10)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)


def test_control_forms_batched_and_refused():
    rt = runtime()
    scs = [scenes.control_forms(seed=6000 + k) for k in range(3)]
    b = rt.Batch(scs)
    singles = [rt.Context(s) for s in scs]
    for _ in range(8):
        b.step()
        for c in singles:
            c.step()
    for i, c in enumerate(singles):
        sg, sc_ = b.state(i), c.state()
        for k in sg:
            assert np.array_equal(sg[k], sc_[k]), (i, k)
    # a spring needs two distinct bodies; a force drive acts on body_b only
    bad = scenes.control_forms()
    bad.drive_body_a = bad.drive_body_a.copy()
    bad.drive_body_a[0] = bad.drive_body_b[0]
    with pytest.raises(rt.NxdError) as e:
        rt.Context(bad)
    assert e.value.status == 7   # NXD_INVALID_ARGUMENT


def test_batch_matches_single_scenes():
    # batched launches (one launch per kernel for all scenes of a group)
    # against the same scenes stepped one context at a time: identical bits;
    # against the oracle: the trajectory tolerance
    scs = scenes.batched_scenes(n_scenes=12)
    rt = runtime()
    b = rt.Batch(scs)
    singles = [rt.Context(s) for s in scs]
    ows = [refcpu.OracleWorld(s) for s in scs]
    for _ in range(10):
        b.step()
        for c in singles:
            c.step()
        for o in ows:
            o.step()
    assert 1 <= b.groups() <= len(scs)
    for i, (s, c, o) in enumerate(zip(scs, singles, ows)):
        sg, sc_, so = b.state(i), c.state(), o.state()
        for k in sg:
            assert np.array_equal(sg[k], sc_[k]), (i, k)
        assert b.diagnostics(i)["status"] == 0
        assert np.abs(sg["position"] - so["position"]).max() <= 1e-6
        assert quat_angle(sg["orientation"], so["orientation"]).max() <= 1e-6


def test_scene_file_fixture():
    # a scene file in the reference's schema (Newmark, allowed contact pairs
    # with friction overrides, hinge + angle limit + velocity drive)
    import os
    from nexdynipc_b200 import sceneio
    fixture = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scene_contact_hinge.json")
    sc, cfg = sceneio.load_scene(fixture)
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    cg = ctx.detect_contacts()
    co, _ = ow.detect_contacts()
    assert len(cg) > 0
    contacts_equal(cg, co)
    wp, wr, _ = run_pair(sc, 20, check_every=5)
    assert wp <= 1e-6 and wr <= 1e-6, (wp, wr)
    # a pair list without Ground-Cube drops those contacts on the device too
    sc2, _ = sceneio.load_scene(fixture)
    sc2.contact_pairs = np.array([[11, 13]], dtype=np.int32)
    sc2.contact_pair_friction = np.array([0.6])
    assert len(runtime().Context(sc2).detect_contacts()) == 0


def test_scene_file_run_writes_reference_csv(tmp_path):
    import os
    from nexdynipc_b200 import sceneio
    fixture = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scene_contact_hinge.json")
    sc, cfg, out = sceneio.run(fixture, output_dir=str(tmp_path))
    d = sceneio.read_state_csv(out.path)
    frames = int(d["frame_idx"].max())
    assert frames == 20                                   # t < 0.1 with dt 0.005
    ow = refcpu.OracleWorld(sc)
    for _ in range(frames):
        ow.step(cfg.dt)
    last = d["frame_idx"] == frames
    assert np.abs(d["pos_y"][last] - ow.state()["position"][:, 1]).max() <= 1e-6


def test_diff_batched_jacobian_matches_oracle():
    # the differentiable-rollout Jacobian from the device batch against the
    # same central differences stepped by the oracle
    from nexdynipc_b200 import diff

    def oracle_runner(worlds, steps):
        out = []
        for w in worlds:
            ow = refcpu.OracleWorld(w)
            for _ in range(steps):
                ow.step()
            out.append(ow.state())
        return out

    sc = scenes.diff_scene()
    spec = diff.ParamSpec(["velocity", "mass", "friction"], bodies=[1, 6])
    theta = spec.get(sc)
    yg, Jg = diff.rollout_jacobian(sc, spec, theta, 8, [1, 6])
    yo, Jo = diff.rollout_jacobian(sc, spec, theta, 8, [1, 6], runner=oracle_runner)
    assert np.abs(yg - yo).max() <= 1e-10
    assert np.abs(Jg - Jo).max() <= 1e-4 * max(1.0, np.abs(Jo).max())
