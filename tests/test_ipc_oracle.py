"""CPU checks of the primitive-level contact model's oracle (full IPC).

The reference has no such model; its arithmetic follows the published method
(Li et al. 2020 IPC, Li et al. 2021 additive CCD) and is shared with the
kernels, so each part is checked here by an independent method:
distances against a constrained minimisation, derivatives against central
finite differences, the subspace PSD projection against a full 12x12
eigen-projection, additive CCD against dense sampling of the trajectory, and
the candidate sets against a brute-force box test.
"""
import numpy as np
import pytest
from scipy.optimize import minimize

from nexdynipc_b200 import scenes
from oracle import refcpu

PT, EE = 0, 1


def brute_dist2(kind, X):
    X = X.reshape(4, 3)
    if kind == PT:
        p, a, b, c = X
        f = lambda u: np.sum((p - (a + u[0] * (b - a) + u[1] * (c - a))) ** 2)
        cons = [{"type": "ineq", "fun": lambda u: 1.0 - u[0] - u[1]}]
        best = np.inf
        for u0 in ([0.2, 0.2], [0.9, 0.05], [0.05, 0.9], [0.0, 0.0]):
            r = minimize(f, u0, bounds=[(0, 1), (0, 1)], constraints=cons, method="SLSQP",
                         options={"ftol": 1e-16, "maxiter": 500})
            best = min(best, r.fun)
        return best
    a0, a1, b0, b1 = X
    f = lambda u: np.sum((a0 + u[0] * (a1 - a0) - b0 - u[1] * (b1 - b0)) ** 2)
    best = np.inf
    for u0 in ([0.5, 0.5], [0.0, 0.0], [1.0, 1.0], [0.0, 1.0], [1.0, 0.0]):
        r = minimize(f, u0, bounds=[(0, 1), (0, 1)], method="L-BFGS-B", options={"ftol": 1e-16, "gtol": 1e-14})
        best = min(best, r.fun)
    return best


def random_pair(rng, kind, dist):
    """Four points whose primitives are about `dist` apart."""
    if kind == PT:
        tri = rng.normal(size=(3, 3))
        n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        n /= np.linalg.norm(n)
        w = rng.dirichlet([1, 1, 1]) * rng.uniform(0.3, 1.6) - rng.uniform(0, 0.3)
        p = tri[0] + w[1] * (tri[1] - tri[0]) + w[2] * (tri[2] - tri[0]) + dist * n
        return np.vstack([p, tri]).reshape(12)
    a = rng.normal(size=(2, 3))
    d = a[1] - a[0]
    m = 0.5 * (a[0] + a[1]) + rng.uniform(-0.8, 0.8) * d
    e = np.cross(d, rng.normal(size=3))
    e /= np.linalg.norm(e)
    off = np.cross(d, e)
    off /= np.linalg.norm(off)
    c = m + dist * off
    half = rng.uniform(0.2, 1.0) * e
    return np.vstack([a, c - half, c + half]).reshape(12)


def cases(n=40, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = i % 2
        out.append((kind, random_pair(rng, kind, rng.uniform(0.05, 0.4))))
    return out


@pytest.mark.parametrize("kind,X", cases())
def test_distance_matches_constrained_minimum(kind, X):
    d2 = refcpu.ipc_dist2(kind, X)
    ref = brute_dist2(kind, X)
    assert d2 == pytest.approx(ref, rel=1e-7, abs=1e-12)


def test_types_cover_every_region():
    seen = {PT: set(), EE: set()}
    for kind, X in cases(400, seed=11):
        seen[kind].add(refcpu.ipc_pair(kind, X, 1.0, 1.0)["type"])
    rng = np.random.default_rng(12)
    for _ in range(400):   # points all around a triangle, projections in (-1, 2)^2
        tri = rng.normal(size=(3, 3))
        n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        u, v = rng.uniform(-1, 2, 2)
        p = tri[0] + u * (tri[1] - tri[0]) + v * (tri[2] - tri[0]) + rng.uniform(-0.3, 0.3) * n
        seen[PT].add(refcpu.ipc_pair(PT, np.vstack([p, tri]).reshape(12), 1.0, 1.0)["type"])
        seen[EE].add(refcpu.ipc_pair(EE, rng.normal(size=12), 1.0, 1.0)["type"])   # two random segments
    assert seen[PT] == set(range(7))
    assert seen[EE] == set(range(9))


@pytest.mark.parametrize("kind,X", cases(24, seed=3))
def test_gradient_and_hessian_finite_differences(kind, X):
    dhat, kappa = 0.5, 1.0
    o = refcpu.ipc_pair(kind, X, dhat, kappa)
    if not o["d2"] < dhat * dhat:
        pytest.skip("pair outside the barrier support")
    h = 1e-6
    g_fd = np.zeros(12)
    H_fd = np.zeros((12, 12))
    t0 = o["type"]
    for i in range(12):
        xp, xm = X.copy(), X.copy()
        xp[i] += h
        xm[i] -= h
        op, om = refcpu.ipc_pair(kind, xp, dhat, kappa), refcpu.ipc_pair(kind, xm, dhat, kappa)
        if op["type"] != t0 or om["type"] != t0:
            pytest.skip("pair within one FD step of a type boundary")
        g_fd[i] = (op["e"] - om["e"]) / (2 * h)
        H_fd[:, i] = (op["g"] - om["g"]) / (2 * h)
    scale = max(np.abs(o["g"]).max(), 1e-12)
    assert np.abs(o["g"] - g_fd).max() <= 1e-6 * scale
    hs = max(np.abs(o["H_raw"]).max(), 1e-12)
    assert np.abs(o["H_raw"] - H_fd).max() <= 1e-5 * hs


@pytest.mark.parametrize("kind,X", cases(40, seed=5))
def test_subspace_projection_equals_full_projection(kind, X):
    o = refcpu.ipc_pair(kind, X, 0.5, 1.0)
    Hs, Hf = o["H_sub"], o["H_full"]
    scale = max(np.abs(o["H_raw"]).max(), 1e-300)
    assert np.abs(Hs - Hf).max() <= 1e-9 * scale
    assert np.abs(Hs - Hs.T).max() <= 1e-12 * scale
    ev = np.linalg.eigvalsh(0.5 * (Hs + Hs.T))
    assert ev.min() >= -1e-10 * scale


def test_barrier_values():
    # b(s) = -kappa (s - sh)^2 ln(s / sh), zero outside the support
    X = np.array([0, 0.3, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1.0])   # point 0.3 above a triangle's corner region
    o = refcpu.ipc_pair(PT, X, 0.5, 2.0)
    s, sh = o["d2"], 0.25
    assert s == pytest.approx(0.09, rel=1e-14)
    assert o["e"] == pytest.approx(-2.0 * (s - sh) ** 2 * np.log(s / sh), rel=1e-13)
    far = refcpu.ipc_pair(PT, X, 0.2, 2.0)
    assert far["e"] == 0.0 and not far["g"].any()


@pytest.mark.parametrize("seed", range(8))
def test_accd_keeps_the_gap(seed):
    rng = np.random.default_rng(100 + seed)
    for kind in (PT, EE):
        X = random_pair(rng, kind, rng.uniform(0.05, 0.3))
        D = rng.normal(scale=0.5, size=12)
        eta = 0.1
        t, it = refcpu.ipc_accd(kind, X, D, 1.0, eta, 1000)
        d0 = np.sqrt(refcpu.ipc_dist2(kind, X))
        assert 0.0 <= t <= 1.0 and it >= 1
        for tt in np.linspace(0.0, t, 401):
            assert np.sqrt(refcpu.ipc_dist2(kind, X + tt * D)) >= eta * d0 * (1 - 1e-9)


def test_accd_head_on_and_separating():
    X = np.array([0.25, 0.5, 0.25, 0, 0, 0, 1, 0, 0, 0, 0, 1.0])   # point above a triangle's interior
    D = np.zeros(12)
    D[1] = -1.0                                                        # moves through the plane at t = 0.5
    t, _ = refcpu.ipc_accd(PT, X, D, 1.0, 0.1, 1000)
    assert 0.4 < t < 0.5
    D[1] = 1.0                                                         # moves away
    t, _ = refcpu.ipc_accd(PT, X, D, 1.0, 0.1, 1000)
    assert t == 1.0


def test_accd_sliding_contact_advances_many_steps_per_round():
    # a point 1e-4 above a triangle sliding 0.5 across it: the conservative
    # step is ~1.6e-4 of the motion, about 6000 steps to t = 1; a round
    # advances up to 32 of them, so t_max is reached within the cap, and a
    # slow approach through the plane (at t = 0.5) stops short of g = 0.1 d0
    X = np.array([0.25, 1e-4, 0.25, 0, 0, 0, 1, 0, 0, 0, 0, 1.0])
    D = np.zeros(12)
    D[0], D[2] = 0.5, 0.1
    t, rounds = refcpu.ipc_accd(PT, X, D, 1.0, 0.1, 1000)
    assert t == 1.0 and rounds < 200
    D[1] = -2e-4
    t, _ = refcpu.ipc_accd(PT, X, D, 1.0, 0.1, 1000)
    assert 0.44 < t < 0.45
    for tt in np.linspace(0.0, t, 201):
        assert np.sqrt(refcpu.ipc_dist2(PT, X + tt * D)) >= 1e-5 * (1 - 1e-9)


def brute_candidates(sc, x, inflation, ow):
    """Box tests of every (vertex, face) and (edge, edge) pair in numpy."""
    import ctypes as C
    L = refcpu.lib()
    nv, nf, ne = C.c_int64(), C.c_int64(), C.c_int64()
    L.nxo_prim_counts.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 3
    L.nxo_prim_counts(ow.h, C.byref(nv), C.byref(nf), C.byref(ne))
    nv, nf, ne = nv.value, nf.value, ne.value
    vb, fb, fv = np.zeros(nv, np.int32), np.zeros(nf, np.int32), np.zeros((nf, 3), np.int32)
    eb, ev = np.zeros(ne, np.int32), np.zeros((ne, 2), np.int32)
    ip = C.POINTER(C.c_int32)
    L.nxo_prim_topology.argtypes = [C.c_void_p, ip, ip, ip, ip, ip]
    cast = lambda a: a.ctypes.data_as(ip)
    L.nxo_prim_topology(ow.h, cast(vb), cast(fb), cast(fv), cast(eb), cast(ev))
    wv = np.zeros((nv, 3))
    L.nxo_world_vertices_at.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    xa = np.ascontiguousarray(x)
    L.nxo_world_vertices_at(ow.h, xa.ctypes.data, wv.ctypes.data, None)
    fmin, fmax = wv[fv].min(1) - inflation, wv[fv].max(1) + inflation
    pt = []
    for v in range(nv):
        hit = np.all((wv[v] <= fmax) & (fmin <= wv[v]), axis=1) & (fb != vb[v])
        pt += [(v, f) for f in np.nonzero(hit)[0]]
    emin, emax = wv[ev].min(1), wv[ev].max(1)
    ee = []
    for a in range(ne):
        hit = np.all((emin[a] <= emax + inflation) & (emin - inflation <= emax[a]), axis=1) & (eb != eb[a])
        ee += [(a, b) for b in np.nonzero(hit)[0] if b > a]
    return np.array(pt, dtype=np.int32).reshape(-1, 2), np.array(ee, dtype=np.int32).reshape(-1, 2)


def scene_x(sc, rng, jitter):
    x = np.zeros(6 * sc.n_bodies)
    for i in range(sc.n_bodies):
        x[6 * i:6 * i + 3] = sc.position[i] + rng.normal(0, jitter, 3)
        x[6 * i + 3:6 * i + 6] = rng.normal(0, jitter, 3)
    return x


def test_oracle_candidates_equal_brute_force():
    sc = scenes.cube_stack()
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, np.random.default_rng(1), 2e-4)
    for infl in (0.0, 1e-3, 0.05):
        pt, ee = ow.ipc_candidates(x, None, infl)
        bpt, bee = brute_candidates(sc, x, infl, ow)
        assert np.array_equal(pt, bpt), infl
        assert np.array_equal(ee, bee), infl
    assert len(ow.ipc_candidates(x, None, 1e-3)[0]) > 0


def test_oracle_barrier_gradient_finite_differences():
    sc = scenes.cube_stack()
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, np.random.default_rng(2), 1e-4)
    dhat, kappa = 1e-3, 1e4
    e, g, H, npairs, nact = ow.ipc_barrier(x, dhat, kappa)
    assert nact > 0 and e > 0
    h = 1e-9
    rng = np.random.default_rng(3)
    idx = rng.choice(len(x), 12, replace=False)
    for i in idx:
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (ow.ipc_barrier(xp, dhat, kappa, hessian=False)[0] - ow.ipc_barrier(xm, dhat, kappa, hessian=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-4 * max(abs(g).max(), 1e-12), (i, fd, g[i])
    assert np.abs(H - H.T).max() <= 1e-12 * np.abs(H).max()
    assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


def test_oracle_barrier_gradient_exact_under_large_rotation_vectors():
    # Each body's orientation is rewound by Exp(-theta0) and the iterate
    # carries theta0 (|theta0| ~ 0.3 rad): the same world poses, so the
    # contacts stay active, but the rotation derivative is now far from the
    # lever arm; the chained gradient (torque times J_r(theta)) must still
    # equal finite differences of the energy.
    from oracle.ipc_adjoint import quat_mul
    sc = scenes.cube_stack()
    ow = refcpu.OracleWorld(sc)
    rng = np.random.default_rng(4)
    x = scene_x(sc, rng, 1e-4)
    st = sc.initial_state()
    for i in range(sc.n_bodies):
        th0 = rng.normal(0, 0.2, 3)
        a = np.linalg.norm(th0)
        inv = np.concatenate([[np.cos(a / 2)], -np.sin(a / 2) * th0 / a])
        st["orientation"][i] = quat_mul(inv, st["orientation"][i])
        x[6 * i + 3:6 * i + 6] += th0
    ow.set_state(st)
    dhat, kappa = 1e-3, 1e4
    e, g, H, npairs, nact = ow.ipc_barrier(x, dhat, kappa)
    assert nact > 0 and e > 0
    h = 1e-7
    rot = [6 * i + 3 + k for i in range(1, sc.n_bodies) for k in range(3)]
    for i in rng.choice(rot, 12, replace=False):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (ow.ipc_barrier(xp, dhat, kappa, hessian=False)[0] - ow.ipc_barrier(xm, dhat, kappa, hessian=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(abs(g).max(), 1e-12), (i, fd, g[i])


def test_accd_follows_the_rotation_arc():
    # A 0.2 m cube 25 mm above the ground turned by 90 degrees about the
    # horizontal z axis: both end poses are clear of the ground, and
    # so are the chords between them, but half-way the bottom corners swing
    # 16 mm below the ground's top face.  The step bound follows the rigid
    # arc x + t dx, so it stops before the corners get there (first contact
    # of the arc at t = 0.19), with every pose on [0, t] clear.
    sc = scenes.ipc_drop(n_cubes=1)
    ow = refcpu.OracleWorld(sc)
    st = sc.initial_state()
    st["orientation"][1] = [1.0, 0.0, 0.0, 0.0]
    st["position"][1] = [0.0, 0.125, 0.0]
    st["velocity"][1] = 0.0
    st["angular_velocity"][1] = 0.0
    ow.set_state(st)
    n = 6 * sc.n_bodies
    x = np.zeros(n)
    x.reshape(-1, 6)[:, :3] = st["position"]
    dx = np.zeros(n)
    dx[6 + 5] = np.pi / 2
    alpha, npairs = ow.ipc_max_step(x, dx, 0.1)
    assert npairs > 0 and 0.1 < alpha < 0.19, alpha
    lowest = []
    for t in np.linspace(0.0, alpha, 200):
        wv, _ = ow.world_vertices_at(x + t * dx)
        lowest.append(wv[8:, 1].min())                      # the cube's vertices (the ground has 8)
    assert min(lowest) > 0.0
    # with the chord the end poses and every chord point would pass
    wv1, _ = ow.world_vertices_at(x + dx)
    assert wv1[8:, 1].min() > 0.02


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_step_bound_keeps_every_pair_apart_along_the_arc(seed):
    # the step bound's guarantee on the rigid arcs: two settled cubes and the
    # ground moved by a random step with rotations up to ~0.6 rad; at every
    # sampled pose x + t dx, t <= the bound, every swept candidate pair keeps
    # at least eta of its distance at x (distances by brute force over the
    # pair's closest points, evaluated on the posed world vertices)
    sc = scenes.ipc_drop(n_cubes=2)
    ow = refcpu.OracleWorld(sc)
    from nexdynipc_b200 import abi
    p = abi.ipc_params(**scenes.ipc_step_settings())
    for _ in range(25):
        ow.ipc_step(p)
    st = ow.state()
    n = 6 * sc.n_bodies
    x = np.zeros(n)
    x.reshape(-1, 6)[:, :3] = st["position"]
    rng = np.random.default_rng(100 + seed)
    dx = np.zeros(n)
    for b in range(1, sc.n_bodies):
        dx[6 * b:6 * b + 3] = rng.normal(0, 0.03, 3) + np.array([0.0, -0.05, 0.0])
        dx[6 * b + 3:6 * b + 6] = rng.normal(0, 0.35, 3)
    eta = 0.1
    alpha, npairs = ow.ipc_max_step(x, dx, eta)
    assert npairs > 0 and 0.0 < alpha <= 1.0
    pt, ee = ow.ipc_candidates(x, dx, 0.0)
    vb, fb, fv, eb, ev = ow.prim_topology()
    pairs = [(0, [v, *fv[f]]) for v, f in pt] + [(1, [*ev[a], *ev[b]]) for a, b in ee]
    w0, _ = ow.world_vertices_at(x)
    d0 = [np.sqrt(refcpu.ipc_dist2(k, w0[vid])) for k, vid in pairs]
    worst = np.inf
    for t in np.linspace(0.0, alpha, 41):
        wt, _ = ow.world_vertices_at(x + t * dx)
        for (k, vid), dd in zip(pairs, d0):
            worst = min(worst, np.sqrt(refcpu.ipc_dist2(k, wt[vid])) / (eta * dd))
    assert worst >= 1.0 - 1e-9, worst
