"""Scene files in the reference's formats (nexdynipc_b200.sceneio): the
JSON scene + OBJ meshes of SceneLoader::load, the SimulationConfig mapping of
Simulation::run, and StateExporter's CSV columns.  Fixture:
tests/golden/scene_contact_hinge.json (written by make_scene_fixture.py)."""
import json
import math
import os

import numpy as np
import pytest

from nexdynipc_b200 import abi, sceneio
from oracle import refcpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURE = os.path.join(GOLDEN, "scene_contact_hinge.json")


def test_obj_fan_triangulation_and_tokens(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("# comment\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\n"
                 "f 1/1/1 2/2/1 3/3/1 4/4/1\nf 1 2\nf 1 x 3\nf 1 2 3\n")
    V, F = sceneio.load_obj(str(p))
    assert V.shape == (4, 3)
    assert F.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 2]]
    q = tmp_path / "empty.obj"
    q.write_text("v 0 0 0\n")
    assert sceneio.load_obj(str(q)) is None


def test_fixture_scene_mapping():
    sc, cfg = sceneio.load_scene(FIXTURE)
    assert list(sc.body_ids) == [10, 11, 12, 13]
    assert sc.body_names == ["Ground", "Cube", "Anchor", "Link"]
    # meshes: ground and cube and link are 8-vertex boxes, fan-triangulated; the anchor has none
    assert list(np.diff(sc.vertex_offset)) == [8, 8, 0, 8]
    assert list(np.diff(sc.face_offset)) == [12, 12, 0, 12]
    # joints: 2 fixed, the revolute entry (the hinge duplicate differs only in
    # stiffness, so it is skipped by signature), then the angle limit
    assert list(sc.joint_type) == [abi.NXD_JOINT_FIXED, abi.NXD_JOINT_FIXED, abi.NXD_JOINT_HINGE,
                                   abi.NXD_JOINT_ANGLE_LIMIT]
    # default stiffness 1e8 becomes settings.joint_stiffness; the angle limit keeps 1e5
    assert list(sc.joint_stiffness) == [1e6, 1e6, 1e6, 1e5]
    assert sc.joint_params[3][3] == pytest.approx(-30 * math.pi / 180, rel=1e-15)
    assert list(sc.joint_params[0][3:7]) == [1.0, 0.0, 0.0, 0.0]   # orientation [x,y,z,w] -> (w,x,y,z)
    # velocity drive (kv, target, max torque from max_torque_nm)
    assert list(sc.drive_body_a) == [12] and list(sc.drive_body_b) == [13]
    assert list(sc.drive_params[0][3:6]) == [0.8, 1.5, 0.2]
    # settings and the contact block
    s = sc.settings
    assert s.integrator == abi.INTEGRATOR_IMPLICIT_NEWMARK and s.newmark_beta == 0.25 and s.newmark_gamma == 0.5
    assert s.alm_max_iters == 4 and s.dhat == 1e-3 and s.enable_adaptive_barrier == 1
    assert cfg.contact_friction == pytest.approx(0.5) and s.enable_friction == 1 and s.friction_coeff == pytest.approx(0.5)
    assert sc.contact_pairs.tolist() == [[10, 11], [11, 13]]          # the disabled pair is left out
    assert sc.contact_pair_friction.tolist() == [0.4, 0.6]
    assert sc.dt == 0.005 and cfg.max_time == 0.1 and cfg.output_name == "fixture_run"


def _write_scene(tmp_path, doc):
    p = tmp_path / "s.json"
    p.write_text(json.dumps(doc))
    for name in ("ground.obj", "cube.obj", "link.obj"):
        (tmp_path / name).write_text(open(os.path.join(GOLDEN, name)).read())
    return str(p)


def test_unsupported_joint_type_is_refused(tmp_path):
    doc = json.load(open(FIXTURE))
    doc["joints"].append({"type": "gear", "body_a": 12, "body_b": 13})
    with pytest.raises(NotImplementedError, match="gear"):
        sceneio.load_scene(_write_scene(tmp_path, doc))


def test_control_form_entries(tmp_path):
    # SceneLoader.cpp:274-446: key fallbacks, defaults, skipped entries and the
    # load order of World::forms ("joints" before "constraints", where the
    # fixture's velocity drive is)
    doc = json.load(open(FIXTURE))
    doc["joints"] += [
        {"type": "damped_spring", "body_a": 12, "body_b": 13, "stiffness_npm": 10.0, "rest_length": 0.2,
         "damping_nspm": 0.5},
        {"type": "damped_spring", "body_a": 99, "body_b": 13, "stiffness_npm": 1.0},     # ignored
        {"type": "position_drive", "body_a": -1, "body_b": 11, "axis": [0, 2, 0], "stiffness": 30.0,
         "target_position_m": 0.4, "max_force_n": 5.0, "deadzone_m": 0.01},
        {"type": "linear_velocity_drive", "body_a": 12, "body_b": 13, "axis": [1, 0, 0],
         "target_velocity": -0.3, "delay_mps": 0.02, "delay_seconds": 0.1},
        {"type": "force_drive", "body_b": 11, "axis": [3, 0, 4], "force_magnitude": 10.0, "torque": [0, 0.1, 0]},
        {"type": "force_drive", "body": 77, "force": [1, 2, 3]},                          # ignored
    ]
    sc, _ = sceneio.load_scene(_write_scene(tmp_path, doc))
    assert list(sc.drive_kind) == [abi.NXD_DRIVE_DAMPED_SPRING, abi.NXD_DRIVE_POSITION,
                                   abi.NXD_DRIVE_LINEAR_VELOCITY, abi.NXD_DRIVE_FORCE, abi.NXD_DRIVE_ANGULAR_VELOCITY]
    assert list(sc.drive_body_a) == [12, -1, 12, -1, 12] and list(sc.drive_body_b) == [13, 11, 13, 11, 13]
    assert list(sc.drive_params[0][:3]) == [0.2, 10.0, 0.5]
    assert list(sc.drive_params[1][3:7]) == [30.0, 0.4, 5.0, 0.01]
    assert list(sc.drive_params[2][3:8]) == [100.0, -0.3, 0.0, 0.02, 0.1]     # kv defaults to 100
    assert list(sc.drive_params[3][:6]) == [0.6 * 10.0, 0.0, 0.8 * 10.0, 0.0, 0.1, 0.0]
    # the oracle builds and steps the scene
    ow = refcpu.OracleWorld(sc)
    for _ in range(3):
        ow.step()
    assert np.isfinite(ow.state()["position"]).all()


def test_state_csv_columns_and_precision(tmp_path):
    sc, cfg = sceneio.load_scene(FIXTURE)
    w = sceneio.StateWriter(str(tmp_path), "out", sc)
    rng = np.random.default_rng(0)
    n = sc.n_bodies
    st = {"position": rng.normal(size=(n, 3)), "orientation": rng.normal(size=(n, 4)),
          "velocity": rng.normal(size=(n, 3)), "linear_acceleration": rng.normal(size=(n, 3)),
          "angular_velocity": rng.normal(size=(n, 3)), "angular_acceleration": rng.normal(size=(n, 3))}
    w.frame(0, 0.0, st)
    w.frame(1, 0.005, st)
    w.kpi(0, 0.0, 0.0, 0.0, 0.0, 0.0)
    w.kpi(1, 0.005, 0.1, 0.2, 0.3, 0.4)
    lines = open(tmp_path / "out.csv").read().splitlines()
    assert lines[0] == ("frame_idx,time,body_id,body_name,pos_x,pos_y,pos_z,qx,qy,qz,qw,vx,vy,vz,ax,ay,az,"
                        "wx,wy,wz,alphax,alphay,alphaz")
    assert len(lines) == 1 + 2 * n
    d = sceneio.read_state_csv(str(tmp_path / "out.csv"))
    assert np.array_equal(d["pos_x"][:n], st["position"][:, 0])          # 17 digits round-trip exactly
    assert np.array_equal(d["qw"][:n], st["orientation"][:, 0])
    assert np.array_equal(d["alphaz"][n:], st["angular_acceleration"][:, 2])
    assert d["body_name"][:n] == ["Ground", "Cube", "Anchor", "Link"]
    k = open(tmp_path / "out_kpi.csv").read().splitlines()
    assert k[0] == "frame_idx,time,V_w,T_sat,R_dual,max_constraint_violation" and k[2].startswith("1,0.005")


def test_allowed_pairs_filter_contacts_in_the_oracle():
    sc, _ = sceneio.load_scene(FIXTURE)
    ow = refcpu.OracleWorld(sc)
    c, _ = ow.detect_contacts()
    assert len(c) > 0 and set(zip(c["body_a"], c["body_b"])) <= {(0, 1), (1, 0)}
    # without the Ground-Cube pair in the list no contact remains
    sc.contact_pairs = np.array([[11, 13]], dtype=np.int32)
    sc.contact_pair_friction = np.array([0.6])
    c2, _ = refcpu.OracleWorld(sc).detect_contacts()
    assert len(c2) == 0
    # the oracle steps the scene
    for _ in range(5):
        ow.step()
    assert np.isfinite(ow.state()["position"]).all()
