"""Writes the scene-file fixture used by tests/test_sceneio.py and
tests/test_gpu_parity.py: a JSON scene in the reference's schema
(SceneLoader::load) with two OBJ meshes.  The scene is synthetic: a fixed
ground box, a unit-density cube resting dhat/2 above it, and a link hinged to
a fixed anchor with an angle limit and a torque-limited velocity drive;
Newmark integration, an allowed contact pair list with friction overrides, a
duplicated joint entry and the deprecated 'revolute' alias.

    python tests/golden/make_scene_fixture.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def box_obj(path, hx, hy, hz):
    v = [(sx * hx, sy * hy, sz * hz) for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
    # quads as 'f' lines (fan-triangulated by the loader), some with v/vt/vn tokens
    quads = [(1, 2, 4, 3), (5, 7, 8, 6), (1, 5, 6, 2), (3, 4, 8, 7), (1, 3, 7, 5), (2, 6, 8, 4)]
    with open(path, "w") as f:
        f.write("# box %g x %g x %g\n" % (2 * hx, 2 * hy, 2 * hz))
        for x in v:
            f.write("v %.17g %.17g %.17g\n" % x)
        for k, q in enumerate(quads):
            if k % 2:
                f.write("f " + " ".join("%d/%d/%d" % (i, i, i) for i in q) + "\n")
            else:
                f.write("f %d %d %d %d\n" % q)


def main():
    box_obj(os.path.join(HERE, "ground.obj"), 2.0, 0.25, 2.0)
    box_obj(os.path.join(HERE, "cube.obj"), 0.1, 0.1, 0.1)
    box_obj(os.path.join(HERE, "link.obj"), 0.02, 0.1, 0.02)
    m = 1000.0 * 0.2 ** 3
    ic = m * (0.2 ** 2 + 0.2 ** 2) / 12.0
    ml = 1000.0 * 0.04 * 0.2 * 0.04
    il = [[ml * (0.2 ** 2 + 0.04 ** 2) / 12, 0, 0], [0, ml * (0.04 ** 2 + 0.04 ** 2) / 12, 0],
          [0, 0, ml * (0.2 ** 2 + 0.04 ** 2) / 12]]
    scene = {
        "case_name": "fixture_contact_hinge",
        "bodies": [
            {"id": 10, "name": "Ground", "mass": 8000.0, "position": [0.0, -0.25, 0.0],
             "inertia": [[1e4, 0, 0], [0, 1e4, 0], [0, 0, 1e4]], "mesh": "ground.obj"},
            {"id": 11, "name": "Cube", "mass": m, "position": [0.3, 0.1005, -0.2],
             "inertia": [[ic, 0, 0], [0, ic, 0], [0, 0, ic]], "mesh": "cube.obj"},
            {"id": 12, "name": "Anchor", "mass": 1.0, "position": [-0.5, 0.8, 0.0]},
            {"id": 13, "name": "Link", "mass": ml, "position": [-0.4, 0.8, 0.0], "inertia": il,
             "mesh": "link.obj"},
        ],
        "joints": [
            {"type": "fixed", "body": 10, "position": [0.0, -0.25, 0.0], "orientation": [0, 0, 0, 1]},
            {"type": "fixed", "body": 12, "position": [-0.5, 0.8, 0.0]},
            {"type": "revolute", "body_a": 12, "body_b": 13, "anchor_a": [0, 0, 0], "anchor_b": [-0.1, 0, 0],
             "axis_a": [0, 0, 1], "axis_b": [0, 0, 1]},
            {"type": "hinge", "body_a": 12, "body_b": 13, "anchor_a": [0, 0, 0], "anchor_b": [-0.1, 0, 0],
             "axis_a": [0, 0, 1], "axis_b": [0, 0, 1], "stiffness": 5e4},
        ],
        "constraints": [
            {"type": "angle_limit", "body_a": 12, "body_b": 13, "axis": [0, 0, 1], "min_angle_deg": -30.0,
             "max_angle_deg": 30.0},
            {"type": "angular_velocity_drive", "body_a": 12, "body_b": 13, "axis": [0, 0, 1],
             "target_velocity_radps": 1.5, "kv": 0.8, "max_torque_nm": 0.2},
        ],
        "settings": {"dt": 0.005, "max_time": 0.1, "integrator_type": "ImplicitNewmark", "newmark_beta": 0.25,
                     "newmark_gamma": 0.5, "joint_stiffness": 1e6, "alm_max_iters": 4,
                     "output_name": "fixture_run"},
        "interactions": {"contact": {
            "global_params": {"default_contact_thickness": 1e-3},
            "pairs": [{"object1": "Ground", "object2": "Cube", "friction": 0.4},
                      {"object1": 11, "object2": 13, "friction": 0.6},
                      {"object1": "Ground", "object2": "Link", "enabled": False, "friction": 0.9}]}},
    }
    with open(os.path.join(HERE, "scene_contact_hinge.json"), "w") as f:
        json.dump(scene, f, indent=1)


if __name__ == "__main__":
    main()
