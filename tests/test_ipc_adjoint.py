"""Adjoint of the full-IPC step (nexdynipc_b200/adjoint.py over
nxd_ipc_adjoint) on the CPU: the chain over steps with checkpoint-and-
recompute, driven by the oracle's step and the CPU restatement of the step
adjoint (oracle/ipc_adjoint.py), against central finite differences of the
oracle's rollout.  Finite differences of a rollout with a stiff barrier are
only as good as the forward solve's convergence (about 1e-10 m here), so the
step is h = 1e-4 (velocities in m/s, relative for masses); the gradient is
checked to 1e-4 of its largest component.  The exact step Jacobian is
checked to be symmetric (it is the Hessian of the step energy)."""
import dataclasses

import numpy as np
import pytest

from nexdynipc_b200 import abi, adjoint, scenes
from oracle import refcpu
from oracle import ipc_adjoint as cpu_adj


def small_scene(n=3, seed=5000):
    rng = np.random.default_rng(seed)
    sb = scenes.SceneBuilder("adjoint_small")
    gv, gf = scenes.box_mesh(1.0, 0.1, 1.0)
    g = sb.add_body(gv, gf, (0.0, -0.1, 0.0))
    sb.fix(g, stiffness=1e5)
    iv, if_ = scenes.icosphere(1)
    for i in range(n):
        sb.add_body(iv * 0.1, if_, (-0.3 + 0.3 * i, 0.102 + 0.01 * rng.random(), 0.0),
                    quat=scenes.random_quaternion(rng), vel=rng.normal(0, 0.3, size=3), omega=rng.normal(0, 2, size=3))
    s = scenes._settings(1e-3, 0.0)
    s.enable_adaptive_barrier = 0
    s.enable_friction = 0
    return sb.build(s, dt=1e-2, steps=10)


PARAMS = abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-12, newton_max_iters=100, ls_max_iters=40)


def loss_and_grads(sc, tgt_p, tgt_q, steps, k=4):
    adj = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa)
    ow = refcpu.OracleWorld(sc)
    r = adjoint.IpcRollout(sc, PARAMS, checkpoint_every=k, ctx=ow, adjoint_fn=lambda st, xs, xb: adj(st, xs, xb, sc.dt))
    T = r.forward(steps)
    L = float(((T["position"] - tgt_p) ** 2).sum() + ((T["orientation"] - tgt_q) ** 2).sum())
    g = r.backward(2 * (T["position"] - tgt_p), 2 * (T["orientation"] - tgt_q))
    return L, g


def rollout_loss(sc, tgt_p, tgt_q, steps):
    ow = refcpu.OracleWorld(sc)
    for _ in range(steps):
        ow.ipc_step(PARAMS)
    T = ow.state()
    return float(((T["position"] - tgt_p) ** 2).sum() + ((T["orientation"] - tgt_q) ** 2).sum())


def test_rollout_adjoint_matches_finite_differences():
    sc = small_scene()
    steps = 10
    rng = np.random.default_rng(1)
    ow = refcpu.OracleWorld(sc)
    for _ in range(steps):
        ow.ipc_step(PARAMS)
    T = ow.state()
    tgt_p = T["position"] + rng.normal(0, 0.01, T["position"].shape)
    tgt_q = T["orientation"] + rng.normal(0, 0.01, T["orientation"].shape)
    L, g = loss_and_grads(sc, tgt_p, tgt_q, steps)
    h = 1e-4
    checks = []
    for b, k in ((1, 0), (1, 1), (2, 1), (3, 2)):
        vp, vm = sc.velocity.copy(), sc.velocity.copy()
        vp[b, k] += h
        vm[b, k] -= h
        fd = (rollout_loss(adjoint.with_parameters(sc, velocity=vp), tgt_p, tgt_q, steps)
              - rollout_loss(adjoint.with_parameters(sc, velocity=vm), tgt_p, tgt_q, steps)) / (2 * h)
        checks.append((g["velocity"][b, k], fd))
    for b in (1, 3):
        hm = h * sc.mass[b]
        mp, mm = sc.mass.copy(), sc.mass.copy()
        mp[b] += hm
        mm[b] -= hm
        fd = (rollout_loss(adjoint.with_parameters(sc, mass=mp), tgt_p, tgt_q, steps)
              - rollout_loss(adjoint.with_parameters(sc, mass=mm), tgt_p, tgt_q, steps)) / (2 * hm)
        checks.append((g["mass"][b], fd))
    a = np.array(checks)
    scale = np.abs(a[:, 1]).max()
    assert np.abs(a[:, 0] - a[:, 1]).max() <= 1e-4 * scale, a


def test_step_jacobian_is_symmetric():
    sc = small_scene()
    ow = refcpu.OracleWorld(sc)
    adj = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa)
    checked = 0
    for t in range(8):
        st0 = ow.state()
        ow.ipc_step(PARAMS)
        xs = adjoint.iterate_of(ow.state(), sc.dt)
        r = adj(st0, xs, np.ones(6 * sc.n_bodies), sc.dt)
        K = r["K"]
        assert np.abs(K - K.T).max() <= 1e-9 * np.abs(K).max()
        checked += len(adj.pairs(xs)) > 0
    assert checked > 0


def step_gradient(sc, st0, x):
    """G(x) of the full-IPC step from the start state st0, restated in numpy
    (inertia, gravity, fixed joints) plus the oracle's barrier gradient."""
    n, dt = sc.n_bodies, sc.dt
    s = dt * dt
    m = sc.mass
    Ib = sc.inertia.reshape(n, 3, 3)
    X = x.reshape(n, 6)
    g = np.zeros((n, 6))
    g[:, :3] = m[:, None] * (X[:, :3] - (st0["position"] + dt * st0["velocity"])) - s * m[:, None] * cpu_adj.GRAVITY
    g[:, 3:] = np.einsum("bij,bj->bi", Ib, X[:, 3:] - dt * st0["angular_velocity"])
    jp = np.asarray(sc.joint_params).reshape(-1, 16)
    for j in range(len(sc.joint_type)):
        a = int(sc.joint_body_a[j])
        tt = cpu_adj.quat_log(cpu_adj.quat_mul(jp[j, 3:7], st0["orientation"][a] * np.array([1.0, -1.0, -1.0, -1.0])))
        g[a] += sc.joint_stiffness[j] * np.concatenate([X[a, :3] - jp[j, :3], X[a, 3:] - tt])
    ow = refcpu.OracleWorld(sc)
    ow.set_state(st0)
    e, gb, H, npairs, nact = ow.ipc_barrier(x, PARAMS.dhat, PARAMS.kappa, hessian=False)
    return g.reshape(-1) + s * gb


def test_step_jacobian_matches_finite_differences_of_the_gradient():
    # K, the heart of the adjoint, against central differences of the step
    # gradient at converged iterates with active contacts; and the gradient
    # itself vanishes there (the implicit function theorem's premise)
    sc = scenes.diff_ipc_scene(n_spheres=4)
    ow = refcpu.OracleWorld(sc)
    adj = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa)
    done = 0
    for t in range(13):
        st0 = ow.state()
        ow.ipc_step(PARAMS)
        if t < 10:
            continue
        xs = adjoint.iterate_of(ow.state(), sc.dt)
        K = adj(st0, xs, np.ones(6 * sc.n_bodies), sc.dt)["K"]
        G = step_gradient(sc, st0, xs)
        assert np.abs(G).max() <= 1e-9
        h = 1e-8
        Kfd = np.zeros_like(K)
        for j in range(len(xs)):
            xp, xm = xs.copy(), xs.copy()
            xp[j] += h
            xm[j] -= h
            Kfd[:, j] = (step_gradient(sc, st0, xp) - step_gradient(sc, st0, xm)) / (2 * h)
        assert len(adj.pairs(xs)) > 0
        assert np.abs(K - Kfd).max() <= 1e-6 * np.abs(K).max(), np.abs(K - Kfd).max()
        done += 1
    assert done == 3


# --- lagged friction (one pass: the pairs frozen at the step start) ---------

MU, EPS = 0.4, 1e-5


def params_f(mu=MU):
    return abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-12, newton_max_iters=100, ls_max_iters=40,
                          mu=mu, friction_eps=EPS, friction_iters=1)


def step_gradient_fric(sc, st0, x, mu=MU):
    """step_gradient plus the oracle's friction gradient of the pairs frozen
    at the start state's pose (nxo_ipc_friction with x_lag = that pose)."""
    n = sc.n_bodies
    ow = refcpu.OracleWorld(sc)
    ow.set_state(st0)
    xl = np.zeros(6 * n)
    xl.reshape(n, 6)[:, :3] = st0["position"]
    _, gf, _, nf = ow.ipc_friction(xl, x, PARAMS.dhat, PARAMS.kappa, mu, EPS, hessian=False)
    return step_gradient(sc, st0, x) + sc.dt * sc.dt * gf, nf


def left_rotated(q, phi):
    a = np.linalg.norm(phi)
    dq = np.concatenate([[np.cos(a / 2)], np.sin(a / 2) * phi / a])
    return cpu_adj.quat_mul(dq, q)


def test_friction_step_jacobian_and_start_state_terms():
    # with friction the step Jacobian K is still the exact derivative of G
    # (central differences at converged iterates), and the start state's
    # position and orientation enter G through the frozen pairs as the
    # adjoint's Kps / Kphi say: d G / d p0 = -m I + Kps, d G / d phi = Kphi
    sc = scenes.diff_ipc_scene(n_spheres=4)
    ow = refcpu.OracleWorld(sc)
    adj = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa, mu=MU, eps=EPS)
    P = params_f()
    done = 0
    for t in range(12):
        st0 = ow.state()
        ow.ipc_step(P)
        if t < 10:
            continue
        xs = adjoint.iterate_of(ow.state(), sc.dt)
        r = adj(st0, xs, np.ones(6 * sc.n_bodies), sc.dt)
        G, nf = step_gradient_fric(sc, st0, xs)
        assert nf > 0 and np.abs(G).max() <= 1e-8
        K = r["K"]
        h = 1e-8
        Kfd = np.zeros_like(K)
        for j in range(len(xs)):
            xp, xm = xs.copy(), xs.copy()
            xp[j] += h
            xm[j] -= h
            Kfd[:, j] = (step_gradient_fric(sc, st0, xp)[0] - step_gradient_fric(sc, st0, xm)[0]) / (2 * h)
        assert np.abs(K - Kfd).max() <= 1e-6 * np.abs(K).max(), np.abs(K - Kfd).max()
        n = sc.n_bodies
        for b in range(1, n):
            for k in range(3):
                sp, sm = {kk: np.array(v, copy=True) for kk, v in st0.items()}, {kk: np.array(v, copy=True) for kk, v in st0.items()}
                sp["position"][b, k] += h
                sm["position"][b, k] -= h
                col = (step_gradient_fric(sc, sp, xs)[0] - step_gradient_fric(sc, sm, xs)[0]) / (2 * h)
                want = r["Kps"][:, 3 * b + k].copy()
                want[6 * b + k] -= sc.mass[b]
                assert np.abs(col - want).max() <= 1e-6 * np.abs(K).max(), (b, k, np.abs(col - want).max())
                e = np.zeros(3)
                e[k] = 1.0
                sp = {kk: np.array(v, copy=True) for kk, v in st0.items()}
                sm = {kk: np.array(v, copy=True) for kk, v in st0.items()}
                sp["orientation"][b] = left_rotated(st0["orientation"][b], h * e)
                sm["orientation"][b] = left_rotated(st0["orientation"][b], -h * e)
                col = (step_gradient_fric(sc, sp, xs)[0] - step_gradient_fric(sc, sm, xs)[0]) / (2 * h)
                assert np.abs(col - r["Kphi"][:, 3 * b + k]).max() <= 1e-6 * np.abs(K).max(), (b, k)
        # d G / d mu
        gp = step_gradient_fric(sc, st0, xs, MU * (1 + 1e-6))[0]
        gm = step_gradient_fric(sc, st0, xs, MU * (1 - 1e-6))[0]
        assert np.abs((gp - gm) / (2e-6 * MU) - r["g_mu"]).max() <= 1e-6 * np.abs(r["g_mu"]).max()
        done += 1
    assert done == 2


def test_friction_rollout_adjoint_matches_finite_differences():
    # the rollout gradient with friction: initial velocities and the friction
    # coefficient against central differences of the oracle's rollout
    sc = small_scene()
    steps = 8
    P = params_f()
    rng = np.random.default_rng(2)
    ow = refcpu.OracleWorld(sc)
    for _ in range(steps):
        ow.ipc_step(P)
    T = ow.state()
    tgt_p = T["position"] + rng.normal(0, 0.01, T["position"].shape)
    tgt_q = T["orientation"] + rng.normal(0, 0.01, T["orientation"].shape)

    def rollout(scn, mu):
        o = refcpu.OracleWorld(scn)
        for _ in range(steps):
            o.ipc_step(params_f(mu))
        S = o.state()
        return float(((S["position"] - tgt_p) ** 2).sum() + ((S["orientation"] - tgt_q) ** 2).sum())

    adj = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa, mu=MU, eps=EPS)
    r = adjoint.IpcRollout(sc, P, checkpoint_every=3, ctx=refcpu.OracleWorld(sc),
                           adjoint_fn=lambda st, xs, xb: adj(st, xs, xb, sc.dt))
    T = r.forward(steps)
    g = r.backward(2 * (T["position"] - tgt_p), 2 * (T["orientation"] - tgt_q))
    h = 1e-4
    checks = []
    for b, k in ((1, 0), (2, 2), (3, 0)):
        vp, vm = sc.velocity.copy(), sc.velocity.copy()
        vp[b, k] += h
        vm[b, k] -= h
        fd = (rollout(adjoint.with_parameters(sc, velocity=vp), MU) - rollout(adjoint.with_parameters(sc, velocity=vm), MU)) / (2 * h)
        checks.append((g["velocity"][b, k], fd))
    hm = h * MU
    fd_mu = (rollout(sc, MU + hm) - rollout(sc, MU - hm)) / (2 * hm)
    checks.append((g["friction"], fd_mu))
    a = np.array(checks)
    scale = np.abs(a[:, 1]).max()
    assert np.abs(a[:, 0] - a[:, 1]).max() <= 1e-4 * scale, a


@pytest.mark.parametrize("kind", [0, 1])
def test_friction_pair_derivatives_match_autograd(kind):
    # the analytic derivatives the device adjoint uses (ipc::friction_derivs)
    # against autograd of the torch restatement, over random pairs of every
    # distance type near contact, their points displaced from the lag state
    import torch
    from test_ipc_oracle import random_pair
    rng = np.random.default_rng(11 + kind)
    dhat, kappa, mu, eps = 1e-1, 1e3, 0.4, 1e-3
    types = set()
    for it in range(90):
        Xs = random_pair(rng, kind, rng.uniform(0.01, 0.09))
        if kind == 1 and it % 3:
            # slide edge b (or a) along itself just past an end: the closest
            # points move to that end vertex (edge-vertex, vertex-vertex types)
            Y = Xs.reshape(4, 3)
            lo = 2 if it % 3 == 1 else 0
            dv = Y[lo + 1] - Y[lo]
            frac = (0.55 + rng.uniform(0.0, 0.05)) * (1.0 if it % 2 else -1.0)
            Y[lo:lo + 2] += frac * dv
            if it % 9 == 5:
                Y[2:] += 0.56 * (Y[3] - Y[2])
            Xs = Y.reshape(12)
        X = Xs + rng.normal(0, 2e-3, 12)
        ev = refcpu.ipc_pair(kind, Xs, dhat, kappa)
        if not (ev["d2"] < dhat * dhat):
            continue
        r = refcpu.ipc_friction_derivs(kind, X, Xs, dhat, kappa, mu, eps)
        typ = r["type"]
        types.add(typ)
        fn = lambda a, b_: cpu_adj.friction_force(kind, typ, a, b_, dhat, kappa, mu, eps)
        Xt, Xst = torch.tensor(X.reshape(4, 3)), torch.tensor(Xs.reshape(4, 3))
        g = fn(Xt, Xst).detach().numpy()
        H, Hs = (j.reshape(12, 12).detach().numpy() for j in torch.autograd.functional.jacobian(fn, (Xt, Xst)))
        sc = max(np.abs(H).max(), np.abs(Hs).max())
        assert np.abs(r["g"] - g).max() <= 1e-10 * np.abs(g).max()
        assert np.abs(r["H"] - H).max() <= 1e-10 * sc
        assert np.abs(r["Hs"] - Hs).max() <= 1e-9 * sc, (typ, np.abs(r["Hs"] - Hs).max() / sc)
    assert len(types) >= 3, types
