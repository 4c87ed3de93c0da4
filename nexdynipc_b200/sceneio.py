"""Scene files in the reference's formats.

* load_scene(path): the JSON scene of SceneLoader::load
  (nexdynipc/src/App/SceneLoader.cpp:460-707) with its OBJ meshes
  (load_obj_mesh, :39-109) into a Scene, plus the SimulationConfig of the
  "settings" and "interactions.contact" blocks (:606-707;
  NexDynIPC/App/Simulation.h:19-53), mapped onto the solver settings the way
  Simulation::run does (src/App/Simulation.cpp:14-56).
* StateWriter: the state and KPI CSVs of StateExporter
  (src/App/StateExporter.cpp:13-76), same columns, values written with 17
  significant digits instead of the default stream precision.
* run(path): Simulation::run's loop (t < max_time: step, export frame and
  KPIs) on the device.

Every joint and constraint kind of SceneLoader::parseJoint is loaded: hinge
(and its deprecated alias revolute), spherical, prismatic, cylindrical, fixed,
angle_limit, distance_limit(s), and the control forms angular_velocity_drive,
linear_velocity_drive, position_drive, force_drive and damped_spring (kept in
load order, as World::forms holds them).  Another type raises
NotImplementedError naming it, where the reference prints "Ignoring
unsupported constraint type".
"""
from __future__ import annotations

import dataclasses
import json
import math
import os

import numpy as np

from . import abi
from .scenes import Scene

_DRIVES = {"angular_velocity_drive", "linear_velocity_drive", "position_drive", "force_drive", "damped_spring"}
_SUPPORTED = {"hinge", "revolute", "spherical", "fixed", "angle_limit", "prismatic", "cylindrical",
              "distance_limit", "distance_limits"} | _DRIVES


def _normalized(v):
    """Eigen's normalized(): v / sqrt((x^2 + y^2) + z^2), v itself when zero."""
    x, y, z = (float(t) for t in v)
    n2 = x * x + y * y + z * z
    if n2 > 0.0:
        n = math.sqrt(n2)
        return [x / n, y / n, z / n]
    return [x, y, z]


def _drive_entry(t, entry, index):
    """(kind, body_a id or -1, body_b id, params[8]) of a control-form entry
    (SceneLoader.cpp:274-446), or None where the loader ignores it."""
    q = np.zeros(8)
    g = entry.get
    if t == "force_drive":
        b = int(g("body", g("body_b", -1)))
        if b not in index:
            return None               # "Ignoring force_drive with invalid body id"
        if "force" in entry:
            q[0:3] = _vec(entry["force"])
        elif "axis" in entry:
            fn = float(g("force_n", g("force_magnitude", 0.0)))
            q[0:3] = [a * fn for a in _normalized(entry["axis"])]
        if "torque" in entry:
            q[3:6] = _vec(entry["torque"])
        return abi.NXD_DRIVE_FORCE, -1, b, q
    if t == "damped_spring":
        a, b = int(g("body_a", -1)), int(g("body_b", -1))
        if a not in index or b not in index:
            return None               # "Ignoring damped_spring with invalid body id"
        q[0] = float(g("rest_length_m", g("rest_length", 0.0)))
        q[1] = float(g("stiffness_npm", g("stiffness", 0.0)))
        q[2] = float(g("damping_nspm", g("damping", 0.0)))
        return abi.NXD_DRIVE_DAMPED_SPRING, a, b, q
    a, b = int(entry["body_a"]), int(entry["body_b"])
    if b not in index:
        return None                   # "Ignoring <drive> with invalid body_b id"
    q[0:3] = _vec(entry["axis"])
    if t == "position_drive":
        q[3] = float(g("kp", g("stiffness", 100.0)))
        q[4] = float(g("target_position_m", g("target_position", 0.0)))
        q[5] = float(g("max_force", g("max_force_n", 0.0)))
        q[6] = float(g("deadzone", g("deadzone_m", 0.0)))
        kind = abi.NXD_DRIVE_POSITION
    elif t == "linear_velocity_drive":
        q[3] = float(g("kv", g("stiffness", 100.0)))
        q[4] = float(g("target_velocity_mps", g("target_velocity", 0.0)))
        q[5] = float(g("max_force", g("max_force_n", 0.0)))
        q[6] = float(g("delay", g("delay_mps", 0.0)))
        q[7] = float(g("delay_tau", g("delay_seconds", 0.0)))
        kind = abi.NXD_DRIVE_LINEAR_VELOCITY
    else:
        q[3] = float(g("kv", g("stiffness", 100.0)))
        q[4] = float(g("target_velocity_radps", 0.0))
        q[5] = float(g("max_torque", g("max_torque_nm", 0.0)))
        q[6] = float(g("delay", g("delay_radps", 0.0)))
        q[7] = float(g("delay_tau", g("delay_seconds", 0.0)))
        kind = abi.NXD_DRIVE_ANGULAR_VELOCITY
    return kind, (a if a in index else -1), b, q


def load_obj(path: str):
    """Vertices and triangles of an OBJ file as load_obj_mesh reads it:
    'v x y z' lines, 'f' lines fan-triangulated from their first index (1-based,
    the index before any '/'); faces with an unparsable or negative index are
    skipped.  Returns (V [n,3] float64, F [m,3] int32) or None when either is
    empty."""
    verts, faces = [], []
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            parts = line.split()
            tag = parts[0]
            if tag == "v":
                xyz = [float(t) for t in parts[1:4]]
                xyz += [0.0] * (3 - len(xyz))
                verts.append(xyz)
            elif tag == "f":
                idx = []
                try:
                    for tok in parts[1:]:
                        head = tok.split("/")[0]
                        if not head:
                            raise ValueError(tok)
                        idx.append(int(head) - 1)
                except ValueError:
                    idx = []
                if len(idx) < 3:
                    continue
                for i in range(1, len(idx) - 1):
                    a, b, c = idx[0], idx[i], idx[i + 1]
                    if a < 0 or b < 0 or c < 0:
                        continue
                    faces.append((a, b, c))
    if not verts or not faces:
        return None
    return np.asarray(verts, dtype=np.float64), np.asarray(faces, dtype=np.int32)


@dataclasses.dataclass
class ContactPairConfig:
    body_a: int
    body_b: int
    enabled: bool = True
    friction: float = -1.0


@dataclasses.dataclass
class SimulationConfig:
    """SimulationConfig (NexDynIPC/App/Simulation.h:19-53) defaults."""
    dt: float = 0.01
    max_time: float = 1.0
    output_dir: str = "output"
    output_name: str = "simulation_results"
    integrator_type: str = "ImplicitNewmark"
    newmark_beta: float = 0.25
    newmark_gamma: float = 0.5
    joint_stiffness: float = 1000.0
    alm_max_iters: int = 6
    alm_constraint_tolerance: float = 1e-4
    alm_dual_tolerance: float = 1e-3
    alm_hardening_trigger: float = 2.0
    alm_hardening_ratio: float = 2.0
    kpi_gate_enabled: bool = False
    kpi_v_w_max: float = 0.2
    kpi_t_sat_max: float = 0.01
    kpi_r_dual_max: float = 1e-3
    contact_enabled: bool = True
    contact_thickness: float = 1e-3
    contact_stiffness: float = -1.0
    contact_friction: float = 0.0
    contact_pairs: list = dataclasses.field(default_factory=list)


def _signature(entry: dict) -> str:
    """make_joint_signature (SceneLoader.cpp:125-139): the entry without its
    stiffness, 'revolute' read as 'hinge', as compact sorted-key JSON."""
    if "type" not in entry:
        return ""
    e = dict(entry)
    if e.get("type") == "revolute":
        e["type"] = "hinge"
    e.pop("stiffness", None)
    return json.dumps(e, sort_keys=True, separators=(",", ":"))


def _vec(v, n=3):
    return [float(v[i]) for i in range(n)]


def load_scene(path: str, dt: float | None = None):
    """Scene and SimulationConfig of a JSON scene file (see the module doc)."""
    with open(path) as f:
        doc = json.load(f)
    scene_dir = os.path.dirname(os.path.abspath(path))
    cfg = SimulationConfig()
    ids, names, pos, mass, inertia, meshes = [], [], [], [], [], []
    for b in doc.get("bodies", []):
        ids.append(int(b.get("id", -1)))
        names.append(str(b.get("name", "Body")))
        pos.append(_vec(b["position"]) if "position" in b else [0.0, 0.0, 0.0])
        mass.append(float(b.get("mass", 1.0)))
        inertia.append(np.asarray(b["inertia"], dtype=np.float64).reshape(9) if "inertia" in b else np.eye(3).reshape(9))
        mesh = None
        if isinstance(b.get("mesh"), str):
            rel = b["mesh"]
            p = rel if os.path.isabs(rel) else os.path.join(scene_dir, rel)
            if not os.path.exists(p) and not os.path.isabs(rel):
                p = os.path.join(os.getcwd(), rel)
            mesh = load_obj(p) if os.path.exists(p) else None
        meshes.append(mesh)
    n = len(ids)
    index = {bid: i for i, bid in enumerate(ids)}

    jt, ja, jb, jp, js = [], [], [], [], []
    da, db, dp, dk = [], [], [], []
    seen = set()
    for entry in list(doc.get("joints", [])) + list(doc.get("constraints", [])):
        if "type" not in entry:
            continue
        sig = _signature(entry)
        if sig and sig in seen:
            continue                  # duplicated joint / constraint entry
        seen.add(sig)
        t = entry["type"]
        if t == "revolute":
            t = "hinge"
        if t not in _SUPPORTED:
            raise NotImplementedError(f"joint/constraint type '{t}' is not implemented by the device step "
                                      f"(supported: {sorted(_SUPPORTED)})")
        p = np.zeros(16)
        if t in ("hinge", "spherical"):
            p[0:3], p[3:6] = _vec(entry["anchor_a"]), _vec(entry["anchor_b"])
            if t == "hinge":
                p[6:9], p[9:12] = _vec(entry["axis_a"]), _vec(entry["axis_b"])
            jt.append(abi.NXD_JOINT_HINGE if t == "hinge" else abi.NXD_JOINT_SPHERICAL)
            ja.append(int(entry["body_a"])); jb.append(int(entry["body_b"]))
            js.append(float(entry.get("stiffness", 1e8)))
        elif t in ("prismatic", "cylindrical"):
            p[0:3], p[3:6] = _vec(entry["anchor_a"]), _vec(entry["anchor_b"])
            p[6:9], p[9:12] = _vec(entry["axis_a"]), _vec(entry["axis_b"])
            jt.append(abi.NXD_JOINT_PRISMATIC if t == "prismatic" else abi.NXD_JOINT_CYLINDRICAL)
            ja.append(int(entry["body_a"])); jb.append(int(entry["body_b"]))
            js.append(float(entry.get("stiffness", 1e8)))
        elif t in ("distance_limit", "distance_limits"):
            a, b2 = int(entry.get("body_a", -1)), int(entry.get("body_b", -1))
            if a not in index or b2 not in index:
                continue
            mn = float(entry.get("min_distance_m", entry.get("min_translation_m", 0.0)))
            mx = float(entry.get("max_distance_m", entry.get("max_translation_m", mn)))
            p[0], p[1] = mn, mx
            jt.append(abi.NXD_JOINT_DISTANCE_LIMIT); ja.append(a); jb.append(b2)
            js.append(float(entry.get("stiffness", 1e5)))
        elif t == "fixed":
            p[0:3] = _vec(entry["position"])
            o = entry.get("orientation")
            p[3:7] = [float(o[3]), float(o[0]), float(o[1]), float(o[2])] if o is not None else [1.0, 0.0, 0.0, 0.0]
            jt.append(abi.NXD_JOINT_FIXED); ja.append(int(entry["body"])); jb.append(-1)
            js.append(float(entry.get("stiffness", 1e8)))
        elif t == "angle_limit":
            a, b2 = int(entry["body_a"]), int(entry["body_b"])
            if a not in index or b2 not in index:
                continue              # "Ignoring angle_limit with invalid body id"
            p[0:3] = _vec(entry["axis"])
            p[3] = float(entry.get("min_angle_deg", -180.0)) * math.pi / 180.0
            p[4] = float(entry.get("max_angle_deg", 180.0)) * math.pi / 180.0
            jt.append(abi.NXD_JOINT_ANGLE_LIMIT); ja.append(a); jb.append(b2)
            js.append(float(entry.get("stiffness", 1e5)))
        else:   # control forms
            d = _drive_entry(t, entry, index)
            if d is not None:
                dk.append(d[0]); da.append(d[1]); db.append(d[2]); dp.append(d[3])
            continue
        jp.append(p)

    # settings block (SceneLoader.cpp:619-644)
    st = doc.get("settings", {})
    for key, field in (("dt", "dt"), ("max_time", "max_time"), ("newmark_gamma", "newmark_gamma"),
                       ("newmark_beta", "newmark_beta"), ("joint_stiffness", "joint_stiffness"),
                       ("integrator_type", "integrator_type"), ("output_name", "output_name"),
                       ("output_dir", "output_dir"), ("alm_max_iters", "alm_max_iters"),
                       ("alm_constraint_tolerance", "alm_constraint_tolerance"),
                       ("alm_dual_tolerance", "alm_dual_tolerance"), ("alm_hardening_trigger", "alm_hardening_trigger"),
                       ("alm_hardening_ratio", "alm_hardening_ratio"), ("kpi_gate_enabled", "kpi_gate_enabled"),
                       ("kpi_v_w_max", "kpi_v_w_max"), ("kpi_t_sat_max", "kpi_t_sat_max"),
                       ("kpi_r_dual_max", "kpi_r_dual_max")):
        if key in st:
            setattr(cfg, field, type(getattr(cfg, field))(st[key]))
    # interactions.contact block (SceneLoader.cpp:646-698)
    contact = doc.get("interactions", {}).get("contact")
    if contact is not None:
        cfg.contact_enabled = True
        gp = contact.get("global_params", {})
        if "default_contact_thickness" in gp:
            cfg.contact_thickness = float(gp["default_contact_thickness"])
        if "min_contact_stiffness" in gp:
            cfg.contact_stiffness = float(gp["min_contact_stiffness"])
        by_name = {nm: bid for nm, bid in zip(names, ids)}

        def resolve(v):
            if isinstance(v, bool):
                return -1
            if isinstance(v, int):
                return v
            if isinstance(v, str):
                return by_name.get(v, -1)
            return -1

        for pr in contact.get("pairs", []) if isinstance(contact.get("pairs"), list) else []:
            if "object1" not in pr or "object2" not in pr:
                continue
            pc = ContactPairConfig(resolve(pr["object1"]), resolve(pr["object2"]), bool(pr.get("enabled", True)),
                                   float(pr.get("friction", -1.0)))
            if pc.body_a >= 0 and pc.body_b >= 0:
                cfg.contact_pairs.append(pc)
        mus = [pc.friction for pc in cfg.contact_pairs if pc.enabled and pc.friction >= 0.0]
        if mus:
            cfg.contact_friction = sum(mus) / len(mus)

    # Simulation::run: joints still at the default stiffness take the global one
    js = [cfg.joint_stiffness if k == 1e8 else k for k in js]
    s = settings_from_config(cfg)
    verts, faces, vo, fo = [], [], [0], [0]
    for m in meshes:
        if m is None:
            vo.append(vo[-1]); fo.append(fo[-1])
        else:
            verts.append(m[0]); faces.append(m[1])
            vo.append(vo[-1] + len(m[0])); fo.append(fo[-1] + len(m[1]))
    nj, nd = len(jt), len(db)
    pairs = [(pc.body_a, pc.body_b, pc.friction) for pc in cfg.contact_pairs if pc.enabled]
    q = np.zeros((n, 4))
    q[:, 0] = 1.0
    sc = Scene(
        name=str(doc.get("case_name", os.path.splitext(os.path.basename(path))[0])),
        position=np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(n, 3)),
        orientation=q, velocity=np.zeros((n, 3)), angular_velocity=np.zeros((n, 3)),
        mass=np.asarray(mass, dtype=np.float64), inertia=np.ascontiguousarray(np.asarray(inertia).reshape(n, 9)),
        vertex_offset=np.asarray(vo, dtype=np.int32), face_offset=np.asarray(fo, dtype=np.int32),
        vertices=np.ascontiguousarray(np.concatenate(verts) if verts else np.zeros((0, 3))),
        faces=np.ascontiguousarray(np.concatenate(faces) if faces else np.zeros((0, 3), np.int32)).astype(np.int32),
        joint_type=np.asarray(jt, dtype=np.int32).reshape(nj), joint_body_a=np.asarray(ja, dtype=np.int32).reshape(nj),
        joint_body_b=np.asarray(jb, dtype=np.int32).reshape(nj),
        joint_params=np.ascontiguousarray(np.asarray(jp, dtype=np.float64).reshape(nj, 16)),
        joint_stiffness=np.asarray(js, dtype=np.float64).reshape(nj),
        drive_body_a=np.asarray(da, dtype=np.int32).reshape(nd), drive_body_b=np.asarray(db, dtype=np.int32).reshape(nd),
        drive_params=np.ascontiguousarray(np.asarray(dp, dtype=np.float64).reshape(nd, 8)),
        drive_kind=np.asarray(dk, dtype=np.int32).reshape(nd),
        settings=s, dt=float(cfg.dt if dt is None else dt), steps=int(math.ceil(cfg.max_time / cfg.dt - 1e-12)),
        body_ids=np.asarray(ids, dtype=np.int32), body_names=names,
        contact_pairs=np.asarray([(a, b) for a, b, _ in pairs], dtype=np.int32).reshape(-1, 2) if pairs else None,
        contact_pair_friction=np.asarray([f for _, _, f in pairs], dtype=np.float64) if pairs else None)
    return sc, cfg


def settings_from_config(cfg: SimulationConfig) -> abi.NxdSettings:
    """Simulation::run's IPCSolver set-up (src/App/Simulation.cpp:26-56)."""
    s = abi.default_settings()
    t = cfg.integrator_type
    if t in ("ImplicitEuler", "Euler"):
        s.integrator = abi.INTEGRATOR_IMPLICIT_EULER
    else:   # ImplicitNewmark, Newmark, and unknown names (create() falls back to Newmark)
        s.integrator = abi.INTEGRATOR_IMPLICIT_NEWMARK
        known = t in ("ImplicitNewmark", "Newmark")
        s.newmark_beta = cfg.newmark_beta if known else 0.25
        s.newmark_gamma = cfg.newmark_gamma if known else 0.5
    s.alm_max_iters = max(1, int(cfg.alm_max_iters))
    s.alm_constraint_tol = cfg.alm_constraint_tolerance
    s.alm_dual_tol = cfg.alm_dual_tolerance
    s.alm_hardening_trigger = cfg.alm_hardening_trigger
    s.alm_hardening_ratio = cfg.alm_hardening_ratio
    fixed = cfg.contact_stiffness > 0.0
    s.enable_adaptive_barrier = int(cfg.contact_enabled and not fixed)
    s.dhat = max(1e-9, cfg.contact_thickness)
    if fixed:
        s.contact_stiffness = cfg.contact_stiffness
    s.enable_friction = int(cfg.contact_friction > 0.0)
    s.friction_coeff = cfg.contact_friction
    return s


def _g(v: float) -> str:
    return format(float(v), ".17g")


class StateWriter:
    """StateExporter's two CSVs (<dir>/<name>.csv and <name>_kpi.csv)."""

    HEADER = ("frame_idx,time,body_id,body_name,pos_x,pos_y,pos_z,qx,qy,qz,qw,vx,vy,vz,ax,ay,az,"
              "wx,wy,wz,alphax,alphay,alphaz\n")
    KPI_HEADER = "frame_idx,time,V_w,T_sat,R_dual,max_constraint_violation\n"

    def __init__(self, output_dir: str, output_name: str, scene: Scene):
        os.makedirs(output_dir, exist_ok=True)
        self.path = os.path.join(output_dir, output_name + ".csv")
        self.kpi_path = os.path.join(output_dir, output_name + "_kpi.csv")
        self.ids = list(scene.body_ids) if scene.body_ids is not None else list(range(scene.n_bodies))
        self.names = scene.body_names or ["Body"] * scene.n_bodies

    def frame(self, frame_idx: int, time: float, state: dict):
        with open(self.path, "w" if frame_idx == 0 else "a") as f:
            if frame_idx == 0:
                f.write(self.HEADER)
            for i in range(len(self.ids)):
                p, q = state["position"][i], state["orientation"][i]
                v, a = state["velocity"][i], state["linear_acceleration"][i]
                w, al = state["angular_velocity"][i], state["angular_acceleration"][i]
                row = [str(frame_idx), _g(time), str(int(self.ids[i])), self.names[i]]
                row += [_g(x) for x in (p[0], p[1], p[2], q[1], q[2], q[3], q[0], v[0], v[1], v[2], a[0], a[1], a[2],
                                        w[0], w[1], w[2], al[0], al[1], al[2])]
                f.write(",".join(row) + "\n")

    def kpi(self, frame_idx: int, time: float, v_w: float, t_sat: float, r_dual: float, mcv: float):
        with open(self.kpi_path, "w" if frame_idx == 0 else "a") as f:
            if frame_idx == 0:
                f.write(self.KPI_HEADER)
            f.write(",".join([str(frame_idx)] + [_g(x) for x in (time, v_w, t_sat, r_dual, mcv)]) + "\n")


def read_state_csv(path: str):
    """Rows of a state CSV as a dict of column arrays (names as strings)."""
    import csv
    with open(path) as f:
        rows = list(csv.DictReader(f))
    out = {}
    for k in rows[0].keys() if rows else []:
        col = [r[k] for r in rows]
        out[k] = col if k == "body_name" else np.asarray([float(c) for c in col])
    return out


def run(path: str, output_dir: str | None = None, context=None):
    """Simulation::run (src/App/Simulation.cpp:14-109) on the device: load,
    export frame 0, then step until t >= max_time exporting every frame and
    its KPIs; the KPI gate raises when enabled and exceeded."""
    from .runtime import Context
    sc, cfg = load_scene(path)
    ctx = context or Context(sc)
    out = StateWriter(output_dir or cfg.output_dir, cfg.output_name, sc)
    t, frame = 0.0, 0
    out.frame(frame, t, ctx.state())
    out.kpi(0, t, 0.0, 0.0, 0.0, 0.0)
    frame += 1
    mx = [0.0, 0.0, 0.0]
    while t < cfg.max_time:
        ctx.step(cfg.dt)
        t += cfg.dt
        d = ctx.diagnostics()
        out.frame(frame, t, ctx.state())
        frame += 1
        out.kpi(frame - 1, t, d["last_angular_velocity_error"], d["last_torque_saturation_ratio"],
                d["last_dual_residual"], d["last_max_constraint_violation"])
        mx = [max(mx[0], d["last_angular_velocity_error"]), max(mx[1], d["last_torque_saturation_ratio"]),
              max(mx[2], d["last_dual_residual"])]
    if cfg.kpi_gate_enabled and not (mx[0] <= cfg.kpi_v_w_max and mx[1] <= cfg.kpi_t_sat_max and mx[2] <= cfg.kpi_r_dual_max):
        raise RuntimeError("KPI gate failed: thresholds exceeded")
    return sc, cfg, out
