"""Seeded synthetic scenes for the contact-step workloads.

No dataset is involved: every configuration is generated here from a seed.
Conventions (Y-up, because the reference hard-wires gravity to (0,-9.81,0),
nexdynipc/src/Dynamics/IPCSolver.cpp:142):

  * static geometry is a body held by a FixedJoint (stiffness 1e8);
  * mass and inertia come from uniform density (divergence theorem) for
    closed meshes, and are given explicitly for open shells;
  * mesh vertices are expressed about the body's centre of mass;
  * friction uses a global coefficient (no allowed-pair list);
  * the implicit-Euler integrator is the only one on this path.

Config seeds are 1000*k (+ scene index for the batched set).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import abi

# ---------------------------------------------------------------------------
# Meshes
# ---------------------------------------------------------------------------

def box_mesh(hx: float, hy: float, hz: float):
    v = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]], dtype=np.float64)
    f = np.array([[0, 2, 1], [0, 3, 2],      # -z
                  [4, 5, 6], [4, 6, 7],      # +z
                  [0, 1, 5], [0, 5, 4],      # -y
                  [3, 7, 6], [3, 6, 2],      # +y
                  [0, 4, 7], [0, 7, 3],      # -x
                  [1, 2, 6], [1, 6, 5]],     # +x
                 dtype=np.int32)
    return v, f


def open_box_mesh(hx: float, hy: float, hz: float):
    """Box without its +y face (a hopper): 8 vertices, 10 triangles, normals
    pointing out of the enclosed volume."""
    v, f = box_mesh(hx, hy, hz)
    keep = [i for i in range(12) if i not in (6, 7)]
    return v, f[keep].copy()


def icosphere(subdiv: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int32)


def random_hull(rng: np.random.Generator, npts: int = 64):
    from scipy.spatial import ConvexHull
    while True:
        p = rng.normal(size=(npts, 3))
        p /= np.linalg.norm(p, axis=1, keepdims=True)
        h = ConvexHull(p)
        if len(h.vertices) == npts:
            break
    f = h.simplices.astype(np.int32).copy()
    # outward orientation
    for i in range(len(f)):
        a, b, c = p[f[i]]
        if np.dot(np.cross(b - a, c - a), a + b + c) < 0:
            f[i] = f[i][[0, 2, 1]]
    return p, f


def bowl_mesh(radius: float, n_lon: int = 32, n_lat: int = 20):
    """Hemispherical shell opening upward (centre of the sphere at origin),
    n_lon*n_lat quads -> 2*n_lon*n_lat triangles (1280 with the defaults)."""
    verts = []
    for i in range(n_lat + 1):
        phi = (math.pi / 2) * i / n_lat          # 0 at the rim, pi/2 at the bottom
        for j in range(n_lon):
            th = 2 * math.pi * j / n_lon
            verts.append((radius * math.cos(phi) * math.cos(th), -radius * math.sin(phi),
                          radius * math.cos(phi) * math.sin(th)))
    faces = []
    for i in range(n_lat):
        for j in range(n_lon):
            a = i * n_lon + j
            b = i * n_lon + (j + 1) % n_lon
            c = (i + 1) * n_lon + j
            d = (i + 1) * n_lon + (j + 1) % n_lon
            faces += [(a, b, d), (a, d, c)]
    return np.array(verts, dtype=np.float64), np.array(faces, dtype=np.int32)


def mass_properties(v: np.ndarray, f: np.ndarray, density: float):
    """Volume, centre of mass and inertia about the COM of a closed, outward
    oriented triangle mesh (signed tetrahedra from the origin)."""
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    d6 = np.einsum("ij,ij->i", a, np.cross(b, c))
    vol = d6.sum() / 6.0
    com = ((a + b + c) * d6[:, None]).sum(0) / (24.0 * vol)
    # second moments of each tetra (0,a,b,c): int x x^T = d6/120 * (sum p p^T + (sum p)(sum p)^T)
    s = a + b + c
    M = np.zeros((3, 3))
    for p in (a, b, c):
        M += np.einsum("i,ij,ik->jk", d6, p, p)
    M += np.einsum("i,ij,ik->jk", d6, s, s)
    M /= 120.0
    mass = density * vol
    cov = density * M - mass * np.outer(com, com)
    inertia = np.trace(cov) * np.eye(3) - cov
    return mass, com, inertia


def quat_from_axis_angle(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    return np.array([math.cos(angle / 2), *(math.sin(angle / 2) * axis)])


def random_quaternion(rng):
    """Uniform random rotation (Shoemake's subgroup algorithm), (w,x,y,z)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    return np.array([q[3], q[0], q[1], q[2]])


def quat_rotate(q, v):
    w, x, y, z = q
    qv = np.array([x, y, z])
    t = 2.0 * np.cross(qv, v)
    return v + w * t + np.cross(qv, t)


# ---------------------------------------------------------------------------
# Scene container
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class Scene:
    name: str
    position: np.ndarray
    orientation: np.ndarray
    velocity: np.ndarray
    angular_velocity: np.ndarray
    mass: np.ndarray
    inertia: np.ndarray
    vertex_offset: np.ndarray
    vertices: np.ndarray
    face_offset: np.ndarray
    faces: np.ndarray
    joint_type: np.ndarray
    joint_body_a: np.ndarray
    joint_body_b: np.ndarray
    joint_params: np.ndarray
    joint_stiffness: np.ndarray
    drive_body_a: np.ndarray
    drive_body_b: np.ndarray
    drive_params: np.ndarray
    settings: abi.NxdSettings
    dt: float
    steps: int
    body_ids: np.ndarray = None                 # RigidBody::id per body (default: the world index)
    body_names: list = None
    contact_pairs: np.ndarray = None            # [n, 2] body ids (IPCSolver::addAllowedContactPair)
    contact_pair_friction: np.ndarray = None    # [n], < 0: no override
    drive_kind: np.ndarray = None               # [n_drives] NXD_DRIVE_* (default: all angular velocity)

    @property
    def n_bodies(self) -> int:
        return int(self.position.shape[0])

    @property
    def n_vertices(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.faces.shape[0])

    def desc(self) -> abi.NxdSceneDesc:
        """NxdSceneDesc viewing this scene's arrays (keep the Scene alive)."""
        self._ids = (np.arange(self.n_bodies, dtype=np.int32) if self.body_ids is None
                     else np.ascontiguousarray(self.body_ids, dtype=np.int32))
        self._zeros3 = np.zeros((self.n_bodies, 3))
        d = abi.NxdSceneDesc()
        d.n_bodies = self.n_bodies
        d.body_ids = abi.iptr(self._ids)
        d.position = abi.dptr(self.position)
        d.orientation = abi.dptr(self.orientation)
        d.velocity = abi.dptr(self.velocity)
        d.angular_velocity = abi.dptr(self.angular_velocity)
        d.linear_acceleration = abi.dptr(self._zeros3)
        d.angular_acceleration = abi.dptr(self._zeros3)
        d.mass = abi.dptr(self.mass)
        d.inertia_body = abi.dptr(self.inertia)
        d.vertex_offset = abi.iptr(self.vertex_offset)
        d.vertices = abi.dptr(self.vertices)
        d.face_offset = abi.iptr(self.face_offset)
        d.faces = abi.iptr(self.faces)
        d.n_joints = int(self.joint_type.shape[0])
        d.joint_type = abi.iptr(self.joint_type)
        d.joint_body_a = abi.iptr(self.joint_body_a)
        d.joint_body_b = abi.iptr(self.joint_body_b)
        d.joint_params = abi.dptr(self.joint_params)
        d.joint_stiffness = abi.dptr(self.joint_stiffness)
        d.n_drives = int(self.drive_body_b.shape[0])
        d.drive_body_a = abi.iptr(self.drive_body_a)
        d.drive_body_b = abi.iptr(self.drive_body_b)
        d.drive_params = abi.dptr(self.drive_params)
        if self.drive_kind is not None and len(self.drive_kind):
            self._dk = np.ascontiguousarray(self.drive_kind, dtype=np.int32)
            d.drive_kind = abi.iptr(self._dk)
        d.settings = self.settings
        if self.contact_pairs is not None and len(self.contact_pairs):
            self._cp = np.ascontiguousarray(self.contact_pairs, dtype=np.int32).reshape(-1, 2)
            fr = (np.full(len(self._cp), -1.0) if self.contact_pair_friction is None
                  else self.contact_pair_friction)
            self._cpf = np.ascontiguousarray(fr, dtype=np.float64)
            d.n_contact_pairs = len(self._cp)
            d.contact_pair_bodies = abi.iptr(self._cp)
            d.contact_pair_friction = abi.dptr(self._cpf)
        return d

    def initial_state(self) -> dict:
        n = self.n_bodies
        return {"position": self.position.copy(), "orientation": self.orientation.copy(),
                "velocity": self.velocity.copy(), "angular_velocity": self.angular_velocity.copy(),
                "linear_acceleration": np.zeros((n, 3)), "angular_acceleration": np.zeros((n, 3))}


class SceneBuilder:
    def __init__(self, name: str):
        self.name = name
        self.bodies = []     # dicts
        self.joints = []     # (type, a, b, params[16], stiffness)
        self.drives = []     # (a, b, params[8], kind)

    def add_body(self, verts, faces, pos, quat=(1, 0, 0, 0), vel=(0, 0, 0), omega=(0, 0, 0),
                 mass=None, inertia=None, density=1000.0, recentre=True):
        verts = np.asarray(verts, dtype=np.float64)
        if mass is None:
            m, com, I = mass_properties(verts, faces, density)
            if recentre:
                verts = verts - com
                pos = np.asarray(pos, dtype=np.float64) + quat_rotate(np.asarray(quat, dtype=np.float64), com)
            mass, inertia = m, I
        self.bodies.append(dict(v=verts, f=np.asarray(faces, dtype=np.int32), p=np.asarray(pos, dtype=np.float64),
                                q=np.asarray(quat, dtype=np.float64), vel=np.asarray(vel, dtype=np.float64),
                                om=np.asarray(omega, dtype=np.float64), m=float(mass),
                                I=np.asarray(inertia, dtype=np.float64).reshape(3, 3)))
        return len(self.bodies) - 1

    def fix(self, b, stiffness=1e8):
        p = np.zeros(16)
        p[0:3] = self.bodies[b]["p"]
        p[3:7] = self.bodies[b]["q"]
        self.joints.append((abi.NXD_JOINT_FIXED, b, -1, p, stiffness))

    def hinge(self, a, b, anchor_a, anchor_b, axis_a, axis_b, stiffness=1e8):
        p = np.zeros(16)
        p[0:3], p[3:6], p[6:9], p[9:12] = anchor_a, anchor_b, axis_a, axis_b
        self.joints.append((abi.NXD_JOINT_HINGE, a, b, p, stiffness))

    def spherical(self, a, b, anchor_a, anchor_b, stiffness=1e8):
        p = np.zeros(16)
        p[0:3], p[3:6] = anchor_a, anchor_b
        self.joints.append((abi.NXD_JOINT_SPHERICAL, a, b, p, stiffness))

    def angle_limit(self, a, b, axis, lo, hi, stiffness=1e5):
        p = np.zeros(16)
        p[0:3] = axis
        p[3], p[4] = lo, hi
        self.joints.append((abi.NXD_JOINT_ANGLE_LIMIT, a, b, p, stiffness))

    def prismatic(self, a, b, anchor_a, anchor_b, axis_a, axis_b, stiffness=1e8):
        p = np.zeros(16)
        p[0:3], p[3:6], p[6:9], p[9:12] = anchor_a, anchor_b, axis_a, axis_b
        self.joints.append((abi.NXD_JOINT_PRISMATIC, a, b, p, stiffness))

    def cylindrical(self, a, b, anchor_a, anchor_b, axis_a, axis_b, stiffness=1e8):
        p = np.zeros(16)
        p[0:3], p[3:6], p[6:9], p[9:12] = anchor_a, anchor_b, axis_a, axis_b
        self.joints.append((abi.NXD_JOINT_CYLINDRICAL, a, b, p, stiffness))

    def distance_limit(self, a, b, min_d, max_d, stiffness=1e5):
        p = np.zeros(16)
        p[0], p[1] = min_d, max_d
        self.joints.append((abi.NXD_JOINT_DISTANCE_LIMIT, a, b, p, stiffness))

    def velocity_drive(self, a, b, axis, kv, v_target, max_torque=0.0, delay=0.0, delay_tau=0.0):
        p = np.zeros(8)
        p[0:3] = axis
        p[3:8] = (kv, v_target, max_torque, delay, delay_tau)
        self.drives.append((a, b, p, abi.NXD_DRIVE_ANGULAR_VELOCITY))

    def linear_velocity_drive(self, a, b, axis, kv, v_target, max_force=0.0, delay=0.0, delay_tau=0.0):
        p = np.zeros(8)
        p[0:3] = axis
        p[3:8] = (kv, v_target, max_force, delay, delay_tau)
        self.drives.append((a, b, p, abi.NXD_DRIVE_LINEAR_VELOCITY))

    def position_drive(self, a, b, axis, kp, target, max_force=0.0, deadzone=0.0):
        p = np.zeros(8)
        p[0:3] = axis
        p[3:7] = (kp, target, max_force, deadzone)
        self.drives.append((a, b, p, abi.NXD_DRIVE_POSITION))

    def force_drive(self, b, force, torque=(0.0, 0.0, 0.0)):
        p = np.zeros(8)
        p[0:3], p[3:6] = force, torque
        self.drives.append((-1, b, p, abi.NXD_DRIVE_FORCE))

    def damped_spring(self, a, b, rest_length, stiffness, damping):
        p = np.zeros(8)
        p[0:3] = (rest_length, stiffness, damping)
        self.drives.append((a, b, p, abi.NXD_DRIVE_DAMPED_SPRING))

    def build(self, settings, dt, steps) -> Scene:
        n = len(self.bodies)
        vo = np.zeros(n + 1, dtype=np.int32)
        fo = np.zeros(n + 1, dtype=np.int32)
        for i, b in enumerate(self.bodies):
            vo[i + 1] = vo[i] + len(b["v"])
            fo[i + 1] = fo[i] + len(b["f"])
        nj = len(self.joints)
        nd = len(self.drives)
        return Scene(
            name=self.name,
            position=np.ascontiguousarray(np.array([b["p"] for b in self.bodies]).reshape(n, 3)),
            orientation=np.ascontiguousarray(np.array([b["q"] for b in self.bodies]).reshape(n, 4)),
            velocity=np.ascontiguousarray(np.array([b["vel"] for b in self.bodies]).reshape(n, 3)),
            angular_velocity=np.ascontiguousarray(np.array([b["om"] for b in self.bodies]).reshape(n, 3)),
            mass=np.array([b["m"] for b in self.bodies], dtype=np.float64),
            inertia=np.ascontiguousarray(np.array([b["I"] for b in self.bodies]).reshape(n, 9)),
            vertex_offset=vo, face_offset=fo,
            vertices=np.ascontiguousarray(np.concatenate([b["v"] for b in self.bodies]).reshape(-1, 3)),
            faces=np.ascontiguousarray(np.concatenate([b["f"] for b in self.bodies]).reshape(-1, 3).astype(np.int32)),
            joint_type=np.array([j[0] for j in self.joints], dtype=np.int32).reshape(nj),
            joint_body_a=np.array([j[1] for j in self.joints], dtype=np.int32).reshape(nj),
            joint_body_b=np.array([j[2] for j in self.joints], dtype=np.int32).reshape(nj),
            joint_params=np.ascontiguousarray(np.array([j[3] for j in self.joints]).reshape(nj, 16)),
            joint_stiffness=np.array([j[4] for j in self.joints], dtype=np.float64).reshape(nj),
            drive_body_a=np.array([d[0] for d in self.drives], dtype=np.int32).reshape(nd),
            drive_body_b=np.array([d[1] for d in self.drives], dtype=np.int32).reshape(nd),
            drive_params=np.ascontiguousarray(np.array([d[2] for d in self.drives]).reshape(nd, 8)),
            drive_kind=np.array([d[3] for d in self.drives], dtype=np.int32).reshape(nd),
            settings=settings, dt=dt, steps=steps)


def _settings(dhat, mu, alm_max_iters=6):
    s = abi.default_settings()
    s.dhat = dhat
    s.enable_friction = 1 if mu > 0 else 0
    s.friction_coeff = mu
    s.alm_max_iters = alm_max_iters
    return s


# ---------------------------------------------------------------------------
# Configurations
# ---------------------------------------------------------------------------

def cube_stack(seed: int = 1000, n_cubes: int = 8, dhat: float = 1e-3, mu: float = 0.5) -> Scene:
    """8 unit cubes (density 1000) stacked with +-5 mm x/z jitter on a static
    10 x 10 x 1 m ground box; dt 1e-2, 100 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("cube_stack")
    gv, gf = box_mesh(5.0, 0.5, 5.0)
    g = sb.add_body(gv, gf, (0.0, -0.5, 0.0))
    sb.fix(g)
    cv, cf = box_mesh(0.5, 0.5, 0.5)
    for i in range(n_cubes):
        jx, jz = rng.uniform(-5e-3, 5e-3, size=2)
        sb.add_body(cv, cf, (jx, 0.5 + i * (1.0 + dhat / 2), jz))
    return sb.build(_settings(dhat, mu), dt=1e-2, steps=100)


def sphere_bowl(seed: int = 2000, n_spheres: int = 64, subdiv: int = 3, dhat: float = 1e-3, mu: float = 0.3) -> Scene:
    """64 seeded icospheres (642 V / 1280 F, radius 0.1*U[0.8,1.2], 2 % radial
    vertex noise) uniform in a 1 m^3 box with uniform random orientations and
    velocities N(0, 0.5), over a static 1280-triangle bowl; dt 5e-3, 200 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("sphere_bowl")
    bv, bf = bowl_mesh(1.2)
    R = 1.2
    b = sb.add_body(bv, bf, (0.0, 0.0, 0.0), mass=1000.0, inertia=np.eye(3) * (2.0 / 3.0) * 1000.0 * R * R)
    sb.fix(b)
    iv, if_ = icosphere(subdiv)
    for _ in range(n_spheres):
        r = 0.1 * rng.uniform(0.8, 1.2)
        noise = 1.0 + 0.02 * rng.uniform(-1.0, 1.0, size=(len(iv), 1))
        v = iv * r * noise
        pos = (rng.uniform(-0.5, 0.5), rng.uniform(-0.3, 0.7), rng.uniform(-0.5, 0.5))
        sb.add_body(v, if_, pos, quat=random_quaternion(rng), vel=rng.normal(0.0, 0.5, size=3))
    return sb.build(_settings(dhat, mu), dt=5e-3, steps=200)


def hopper_chains(seed: int = 3000, n_hulls: int = 1024, n_chains: int = 32, links: int = 8,
                  dhat: float = 5e-4, mu: float = 0.3) -> Scene:
    """1024 convex hulls of 64 seeded unit-sphere points scaled to 0.05 m in a
    1 x 4 x 1 m open-top hopper, plus 32 hinge chains of 8 links (each hinge
    with a +-60 degree angle limit) hanging from fixed anchors beside it;
    dt 5e-3, 2 ALM (lagged-friction) iterations, 100 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("hopper_chains")
    hv, hf = open_box_mesh(0.5, 2.0, 0.5)
    h = sb.add_body(hv, hf, (0.0, 2.0, 0.0), mass=1e4, inertia=np.diag([1e4 * (16 + 1) / 12, 1e4 * 2 / 12, 1e4 * 17 / 12]))
    sb.fix(h)
    per_side = 8
    pitch = 0.125
    layers = (n_hulls + per_side * per_side - 1) // (per_side * per_side)
    k = 0
    for ly in range(layers):
        for ix in range(per_side):
            for iz in range(per_side):
                if k >= n_hulls:
                    break
                p, f = random_hull(rng)
                pos = (-0.4375 + ix * pitch + rng.uniform(-0.01, 0.01), 0.1 + ly * pitch + rng.uniform(-0.01, 0.01),
                       -0.4375 + iz * pitch + rng.uniform(-0.01, 0.01))
                sb.add_body(p * 0.05, f, pos, quat=random_quaternion(rng), vel=rng.normal(0.0, 0.1, size=3))
                k += 1
    # chains: anchor cube + links (boxes 0.02 x 0.1 x 0.02) joined end to end
    lv, lf = box_mesh(0.01, 0.05, 0.01)
    av, af = box_mesh(0.025, 0.025, 0.025)
    half = 0.051
    tilt = math.radians(30.0)
    q = quat_from_axis_angle((0, 0, 1), tilt)
    down = quat_rotate(q, np.array([0.0, -1.0, 0.0]))
    for c in range(n_chains):
        ax = 1.0 + 0.25 * (c % 8)
        az = -0.45 + 0.3 * (c // 8)
        anchor_pos = np.array([ax, 2.5, az])
        a = sb.add_body(av, af, anchor_pos)
        sb.fix(a)
        prev = a
        # hinge 1 mm below the anchor cube's bottom face
        prev_anchor = np.array([0.0, -0.026, 0.0])
        top = anchor_pos + prev_anchor
        for l in range(links):
            centre = top + down * half
            li = sb.add_body(lv, lf, centre, quat=q)
            sb.hinge(prev, li, prev_anchor, (0.0, half, 0.0), (0, 0, 1), (0, 0, 1))
            sb.angle_limit(prev, li, (0, 0, 1), -math.radians(60), math.radians(60))
            prev = li
            prev_anchor = np.array([0.0, -half, 0.0])
            top = centre + down * half
    return sb.build(_settings(dhat, mu, alm_max_iters=2), dt=5e-3, steps=100)


def batched_scenes(seed: int = 4000, n_scenes: int = 256):
    """256 independent scenes, body count floor(exp(U[ln 2, ln 64])) each:
    cubes, icospheres (162 V) and 2-10 link hinge or spherical chains with
    torque-limited velocity drives, over a fixed ground box; dt 1e-2,
    dhat 1e-3, mu ~ U[0.1, 0.8], 100 steps."""
    scenes = []
    iv, if_ = icosphere(2)
    cv, cf = box_mesh(0.05, 0.05, 0.05)
    lv, lf = box_mesh(0.01, 0.04, 0.01)
    for si in range(n_scenes):
        rng = np.random.default_rng(seed + si)
        nb = int(math.floor(math.exp(rng.uniform(math.log(2), math.log(64)))))
        mu = rng.uniform(0.1, 0.8)
        sb = SceneBuilder(f"batched_{si}")
        gv, gf = box_mesh(2.0, 0.1, 2.0)
        g = sb.add_body(gv, gf, (0.0, -0.1, 0.0))
        sb.fix(g)
        count = 1
        slot = 0
        while count < nb:
            kind = rng.integers(0, 3)
            x = -1.5 + 0.35 * (slot % 9)
            z = -1.5 + 0.35 * (slot // 9)
            slot += 1
            if kind == 0:
                sb.add_body(cv, cf, (x, 0.06 + rng.uniform(0.0, 0.3), z), quat=random_quaternion(rng),
                            vel=rng.normal(0, 0.2, size=3))
                count += 1
            elif kind == 1:
                sb.add_body(iv * 0.05, if_, (x, 0.06 + rng.uniform(0.0, 0.3), z), quat=random_quaternion(rng),
                            vel=rng.normal(0, 0.2, size=3))
                count += 1
            else:
                nl = int(min(rng.integers(2, 11), nb - count))
                if nl < 1:
                    break
                spherical = bool(rng.integers(0, 2))
                anchor = sb.add_body(cv * 0.5, cf, (x, 0.9, z))
                sb.fix(anchor)
                count += 1
                prev, prev_anchor = anchor, np.array([0.0, -0.026, 0.0])
                top = np.array([x, 0.9, z]) + prev_anchor
                for _ in range(nl):
                    if count >= nb:
                        break
                    centre = top + np.array([0.0, -0.041, 0.0])
                    li = sb.add_body(lv, lf, centre)
                    if spherical:
                        sb.spherical(prev, li, prev_anchor, (0.0, 0.041, 0.0))
                    else:
                        sb.hinge(prev, li, prev_anchor, (0.0, 0.041, 0.0), (0, 0, 1), (0, 0, 1))
                        sb.velocity_drive(prev, li, (0, 0, 1), kv=0.5, v_target=rng.uniform(-2, 2),
                                          max_torque=0.05)
                    prev, prev_anchor, top = li, np.array([0.0, -0.041, 0.0]), centre + np.array([0.0, -0.041, 0.0])
                    count += 1
        scenes.append(sb.build(_settings(1e-3, mu), dt=1e-2, steps=100))
    return scenes


def control_forms(seed: int = 6000, dhat: float = 1e-3, mu: float = 0.4) -> Scene:
    """Every control form of World::forms on 0.1 m boxes over a static ground
    box: a damped spring from a fixed anchor, a saturating position drive
    with a deadzone to the world and one between two boxes, a torque-limited
    linear velocity drive with a target filter, an angular velocity drive, and
    a force drive with a torque; dt 1e-2, 60 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("control_forms")
    gv, gf = box_mesh(2.0, 0.25, 2.0)
    g = sb.add_body(gv, gf, (0.0, -0.25, 0.0))
    sb.fix(g)
    bv, bf = box_mesh(0.05, 0.05, 0.05)
    anchor = sb.add_body(bv, bf, (0.0, 1.2, 0.0))
    sb.fix(anchor)
    jit = lambda: rng.uniform(-0.02, 0.02, size=3)
    hang = sb.add_body(bv, bf, (0.05, 0.85, 0.02) + jit(), vel=(0.2, 0.0, -0.1))
    slide = sb.add_body(bv, bf, (0.4, 0.05 + dhat / 2, 0.0) + jit() * (1, 0, 1))
    follow = sb.add_body(bv, bf, (0.7, 0.05 + dhat / 2, 0.1) + jit() * (1, 0, 1))
    spin = sb.add_body(bv, bf, (-0.4, 0.05 + dhat / 2, -0.2) + jit() * (1, 0, 1))
    push = sb.add_body(bv, bf, (-0.6, 0.3, 0.3) + jit(), omega=(0.0, 0.5, 0.0))
    sb.damped_spring(anchor, hang, rest_length=0.3, stiffness=400.0, damping=2.0)
    sb.position_drive(-1, slide, (1.0, 0.0, 0.2), kp=60.0, target=0.55, max_force=4.0, deadzone=0.01)
    sb.linear_velocity_drive(slide, follow, (1.0, 0.0, 0.0), kv=0.05, v_target=-0.2, max_force=0.5,
                             delay=0.01, delay_tau=0.05)
    sb.velocity_drive(g, spin, (0.0, 1.0, 0.0), kv=0.002, v_target=0.5, max_torque=0.01)
    sb.force_drive(push, (0.3, 4.0, 0.0), torque=(0.0, 0.0, 0.02))
    sb.position_drive(hang, push, (0.0, 1.0, 0.0), kp=25.0, target=-0.4)
    return sb.build(_settings(dhat, mu), dt=1e-2, steps=60)


def ipc_drop(seed: int = 7000, n_cubes: int = 2, columns: int = 1) -> Scene:
    """Full-IPC configuration: n 0.2 m cubes (8 kg) dropped, tilted and
    jittered, onto a static 2 x 0.2 x 2 m ground box in `columns` stacks on
    a square grid of 0.4 m pitch centred on the origin (cube i in stack
    i % columns, level i // columns), their centres 0.2 m above the ground
    and 0.4 m apart per level (clear of any tilt); cubes above the first
    level start at 1 m/s downward; COM-distance contact forms off
    (enable_adaptive_barrier and friction off), dt 1e-2, 80 steps.  Stepped
    with nxd_ipc_step."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("ipc_drop")
    gv, gf = box_mesh(1.0, 0.1, 1.0)
    g = sb.add_body(gv, gf, (0.0, -0.1, 0.0))
    sb.fix(g)
    cv, cf = box_mesh(0.1, 0.1, 0.1)
    side = int(math.ceil(math.sqrt(columns)))
    for i in range(n_cubes):
        jx, jz = rng.uniform(-0.05, 0.05, size=2)
        q = quat_from_axis_angle(rng.normal(size=3), rng.uniform(0.0, 0.4))
        col, lvl = i % columns, i // columns
        cx, cz = 0.4 * (col % side - 0.5 * (side - 1)), 0.4 * (col // side - 0.5 * (side - 1))
        sb.add_body(cv, cf, (cx + jx, 0.2 + 0.4 * lvl, cz + jz), quat=q, vel=(0.0, -1.0 if lvl else 0.0, 0.0))
    s = _settings(1e-3, 0.0)
    s.enable_adaptive_barrier = 0
    s.enable_friction = 0
    return sb.build(s, dt=1e-2, steps=80)


def ipc_step_settings(solver: int = 0, mu: float = 0.0) -> dict:
    """Keyword arguments of abi.ipc_params for the full-IPC steps run on
    ipc_drop and on sphere_bowl: dhat 1e-3, kappa 1e11, eta 0.1 (the CCD
    bound keeps 90 % of each pair's distance), Newton until |g|_inf < 1e-5
    (or the step below 1e-5 dt) in at most 50 iterations, 30 Armijo trials;
    solver 0 = component LDL^T, 1 = block-Jacobi PCG (500 iterations, 1e-12).
    mu > 0 adds lagged friction with eps 1e-5 m over 2 lagging passes (the
    reference's default eps of 1e-8 m makes the sticking branch 1000x
    stiffer, and Newton then stalls at its iteration limit on the bowl)."""
    return dict(dhat=1e-3, kappa=1e11, eta=0.1, newton_tol=1e-5, newton_max_iters=50, ls_max_iters=30,
                linear_solver=solver, pcg_max_iter=500, pcg_tol=1e-12, mu=mu, friction_eps=1e-5, friction_iters=2)


def diff_scene(seed: int = 5000) -> Scene:
    """16 icospheres (162 V) colliding on a ground box, dt 1e-2, 50 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("diff_spheres")
    gv, gf = box_mesh(2.0, 0.1, 2.0)
    g = sb.add_body(gv, gf, (0.0, -0.1, 0.0))
    sb.fix(g)
    iv, if_ = icosphere(2)
    for i in range(16):
        sb.add_body(iv * 0.1, if_, (-0.6 + 0.4 * (i % 4), 0.12 + 0.05 * rng.random(), -0.6 + 0.4 * (i // 4)),
                    quat=random_quaternion(rng), vel=rng.normal(0, 0.3, size=3))
    return sb.build(_settings(1e-3, 0.3), dt=1e-2, steps=50)


def diff_ipc_scene(seed: int = 5000, n_spheres: int = 16, subdiv: int = 2) -> Scene:
    """The differentiable configuration for the full-IPC step and its
    adjoint: diff_scene's 16 icospheres (162 V) over a ground box, the ground
    held by a FixedJoint of stiffness 1e5 (its sag under the spheres stays
    below 1e-5 m, and the joint does not amplify rounding the way 1e8 does),
    COM-distance contact forms off (nxd_ipc_step), dt 1e-2, 50 steps."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder("diff_ipc_spheres")
    gv, gf = box_mesh(2.0, 0.1, 2.0)
    g = sb.add_body(gv, gf, (0.0, -0.1, 0.0))
    sb.fix(g, stiffness=1e5)
    iv, if_ = icosphere(subdiv)
    for i in range(n_spheres):
        sb.add_body(iv * 0.1, if_, (-0.6 + 0.4 * (i % 4), 0.12 + 0.05 * rng.random(), -0.6 + 0.4 * (i // 4)),
                    quat=random_quaternion(rng), vel=rng.normal(0, 0.3, size=3))
    s = _settings(1e-3, 0.0)
    s.enable_adaptive_barrier = 0
    s.enable_friction = 0
    return sb.build(s, dt=1e-2, steps=50)


def double_pendulum(dt: float = 1e-3, max_time: float = 1.5, inertia_zz=(1.0, 1.0)) -> Scene:
    """The reference's double-pendulum regression case as its scene loader
    builds it (nexdynipc/assets/double_pendulum/double_pendulum.json through
    SceneLoader and Simulation::run): a meshless 1 kg anchor held by a
    FixedJoint at the origin and two meshless 1 kg links with unit inertia at
    (0.5, 0, 0) and (1.5, 0, 0), hinged about z at (0, 0, 0) and (1, 0, 0),
    released at rest; ImplicitNewmark (beta 0.25, gamma 0.5), every joint at
    the file's joint_stiffness 1e7, dt 1e-3, 1.5 s.  inertia_zz sets the
    links' inertia about the hinge axis (the other diagonal entries stay 1)."""
    from .sceneio import SimulationConfig, settings_from_config
    sb = SceneBuilder("double_pendulum")
    ev, ef = np.zeros((0, 3)), np.zeros((0, 3), np.int32)
    sb.add_body(ev, ef, (0.0, 0.0, 0.0), mass=1.0, inertia=np.eye(3))
    for k, x in enumerate((0.5, 1.5)):
        sb.add_body(ev, ef, (x, 0.0, 0.0), mass=1.0, inertia=np.diag([1.0, 1.0, float(inertia_zz[k])]))
    sb.fix(0, stiffness=1e7)
    sb.hinge(0, 1, (0.0, 0.0, 0.0), (-0.5, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, 1.0), stiffness=1e7)
    sb.hinge(1, 2, (0.5, 0.0, 0.0), (-0.5, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, 1.0), stiffness=1e7)
    cfg = SimulationConfig(dt=dt, max_time=max_time, joint_stiffness=1e7)
    return sb.build(settings_from_config(cfg), dt, int(math.ceil(max_time / dt - 1e-12)))


CONFIGS = {
    "cube_stack": cube_stack,
    "sphere_bowl": sphere_bowl,
    "hopper_chains": hopper_chains,
    "diff_spheres": diff_scene,
}
