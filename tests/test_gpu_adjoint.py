"""The device adjoint of the full-IPC step (nxd_ipc_adjoint) against its CPU
restatement (oracle/ipc_adjoint.py, which uses the oracle's independently
written pair Hessian), step by step along a device rollout of the
differentiable configuration, and the device rollout gradient
(nexdynipc_b200/adjoint.py) against central finite differences of device
rollouts, for several parameter sets (initial velocities)."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, adjoint, scenes

pytestmark = pytest.mark.gpu

PARAMS = abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-9, newton_max_iters=100, ls_max_iters=40)


def test_device_step_adjoint_matches_cpu_restatement():
    from nexdynipc_b200 import runtime
    from oracle import ipc_adjoint as cpu_adj
    sc = scenes.diff_ipc_scene(n_spheres=6)
    ctx = runtime.Context(sc)
    cpu = cpu_adj.StepAdjoint(sc, PARAMS.dhat, PARAMS.kappa)
    rng = np.random.default_rng(3)
    checked = 0
    for t in range(14):
        st0 = ctx.state()
        ctx.ipc_step(PARAMS)
        st1 = ctx.state()
        xs = adjoint.iterate_of(st1, sc.dt)
        xb = rng.normal(size=6 * sc.n_bodies)
        d = ctx.ipc_adjoint(st0, xs, xb, PARAMS)
        c = cpu(st0, xs, xb, sc.dt)
        for k in ("lam", "phat_bar", "thetahat_bar", "phi_bar", "mass_bar", "inertia_bar", "joint_mu_bar"):
            ref = np.asarray(c[k])
            assert np.abs(np.asarray(d[k]) - ref).max() <= 1e-8 * max(np.abs(ref).max(), 1e-30), (t, k)
        checked += d["n_active"] > 0
        ctx.set_state(st1)
    assert checked >= 4


def test_device_rollout_gradients_match_finite_differences():
    # A rollout of stiff contacts is piecewise smooth in its parameters: a
    # perturbed run can take another branch (another local minimum of a
    # step, visible as a different sequence of active-pair counts), and a
    # central difference across branches means nothing.  Entries whose
    # perturbed runs leave the base run's branch are not compared (most
    # are).  The rest must agree to 5e-3 of the gradient's largest entry:
    # the forward solve stops at |g| < 1e-9, which leaves the light spheres'
    # rotations determined to about |g| / I (1e-8 rad for I = 0.017 kg m^2),
    # and central differences of the final poses with h = 1e-4 inherit that
    # noise.  (The exact step Jacobian itself is checked against finite
    # differences of the step gradient on the CPU, tests/test_ipc_adjoint.py.)
    from nexdynipc_b200 import runtime
    base = scenes.diff_ipc_scene(n_spheres=4)
    steps = 20
    rng = np.random.default_rng(11)
    ctx = runtime.Context(base)
    fd_ctx = runtime.Context(base)

    def run(sc, tgt_p, tgt_q, fresh=False):
        # velocities are state (set on the same context); masses live in the
        # context, so a mass perturbation needs a context of its own
        c = runtime.Context(sc) if fresh else fd_ctx
        c.set_state(sc.initial_state())
        act = [c.ipc_step(PARAMS)["n_active"] for _ in range(steps)]
        T = c.state()
        return float(((T["position"] - tgt_p) ** 2).sum() + ((T["orientation"] - tgt_q) ** 2).sum()), act

    h = 1e-4
    compared = total = 0
    worst = 0.0
    for ps in range(3):                      # parameter sets: perturbed initial velocities
        v0 = base.velocity + rng.normal(0, 0.05, base.velocity.shape)
        sc = adjoint.with_parameters(base, velocity=v0)
        r = adjoint.IpcRollout(sc, PARAMS, checkpoint_every=5, ctx=ctx)
        T = r.forward(steps)
        branch = [s["n_active"] for s in r.stats]
        tgt_p = T["position"] + rng.normal(0, 0.01, T["position"].shape)
        tgt_q = T["orientation"] + rng.normal(0, 0.01, T["orientation"].shape)
        g = r.backward(2 * (T["position"] - tgt_p), 2 * (T["orientation"] - tgt_q))
        a, f = [], []
        cases = [("velocity", b, k) for b in range(1, sc.n_bodies) for k in range(3)] + [("mass", 1, 0)]
        for kind, b, k in cases:
            total += 1
            if kind == "velocity":
                vp, vm = v0.copy(), v0.copy()
                vp[b, k] += h
                vm[b, k] -= h
                (lp, ap), (lm, am) = (run(adjoint.with_parameters(sc, velocity=vp), tgt_p, tgt_q),
                                      run(adjoint.with_parameters(sc, velocity=vm), tgt_p, tgt_q))
                d, ad = (lp - lm) / (2 * h), g["velocity"][b, k]
            else:
                hm = h * sc.mass[b]
                mp, mm = sc.mass.copy(), sc.mass.copy()
                mp[b] += hm
                mm[b] -= hm
                (lp, ap), (lm, am) = (run(adjoint.with_parameters(sc, mass=mp), tgt_p, tgt_q, fresh=True),
                                      run(adjoint.with_parameters(sc, mass=mm), tgt_p, tgt_q, fresh=True))
                d, ad = (lp - lm) / (2 * hm), g["mass"][b]
            if ap != branch or am != branch:
                continue
            a.append(ad)
            f.append(d)
        a, f = np.array(a), np.array(f)
        compared += len(a)
        err = np.abs(a - f).max() / np.abs(f).max()
        print(f"parameter set {ps}: {len(a)}/{len(cases)} on the base branch, max |adjoint - FD| / max |FD| = {err:.2e}")
        worst = max(worst, err)
    assert compared >= 0.6 * total, (compared, total)
    assert worst <= 5e-3, worst


def test_device_friction_adjoint_matches_cpu_restatement():
    # with lagged friction (one pass, mu 0.4): the device's analytic
    # derivatives of the frozen pairs (ipc::friction_derivs) against the
    # restatement's autograd, through every output, including the step-start
    # positions' and the friction coefficient's adjoints.  Tolerance 1e-6 of
    # each output's largest entry: the sticking stiffness mu lam / eps
    # (~1e6 N/m at eps 1e-5 m) enters K and K_phi, and the outputs are sums of
    # terms that large which cancel to O(1), so two different operation
    # orders differ by more than the frictionless test's 1e-8 (a lost update
    # in the assembly showed as 1e-3).
    from nexdynipc_b200 import runtime
    from oracle import ipc_adjoint as cpu_adj
    mu, eps = 0.4, 1e-5
    P = abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-9, newton_max_iters=100, ls_max_iters=40,
                       mu=mu, friction_eps=eps, friction_iters=1)
    sc = scenes.diff_ipc_scene(n_spheres=6)
    ctx = runtime.Context(sc)
    cpu = cpu_adj.StepAdjoint(sc, P.dhat, P.kappa, mu=mu, eps=eps)
    rng = np.random.default_rng(4)
    checked = 0
    for t in range(14):
        st0 = ctx.state()
        stats = ctx.ipc_step(P)
        st1 = ctx.state()
        xs = adjoint.iterate_of(st1, sc.dt)
        xb = rng.normal(size=6 * sc.n_bodies)
        d = ctx.ipc_adjoint(st0, xs, xb, P)
        c = cpu(st0, xs, xb, sc.dt)
        for k in ("lam", "phat_bar", "thetahat_bar", "phi_bar", "mass_bar", "inertia_bar", "joint_mu_bar", "p0_bar",
                  "friction_mu_bar"):
            ref = np.asarray(c[k])
            assert np.abs(np.asarray(d[k]) - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1e-30), (t, k)
        checked += stats["n_friction"] > 0
        ctx.set_state(st1)
    assert checked >= 4


def test_device_friction_rollout_gradient_matches_finite_differences():
    # the friction coefficient's and initial velocities' gradients of a
    # device rollout with lagged friction (three spheres landing and sliding
    # on a ground box from the first steps, so friction acts on most steps)
    # against central differences of device rollouts on the same branch of
    # active-pair counts; Newton to |g| < 1e-12 as in the CPU test
    from nexdynipc_b200 import runtime
    from test_ipc_adjoint import small_scene
    mu, eps, steps = 0.4, 1e-5, 8

    def params(m):
        return abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-12, newton_max_iters=100, ls_max_iters=40,
                              mu=m, friction_eps=eps, friction_iters=1)

    sc = small_scene()
    ctx = runtime.Context(sc)
    r = adjoint.IpcRollout(sc, params(mu), checkpoint_every=3, ctx=ctx)
    T = r.forward(steps)
    assert sum(s["n_friction"] for s in r.stats) > 0
    branch = [s["n_active"] for s in r.stats]
    rng = np.random.default_rng(2)
    tgt_p = T["position"] + rng.normal(0, 0.01, T["position"].shape)
    tgt_q = T["orientation"] + rng.normal(0, 0.01, T["orientation"].shape)
    g = r.backward(2 * (T["position"] - tgt_p), 2 * (T["orientation"] - tgt_q))
    fd_ctx = runtime.Context(sc)

    def loss(scn, m):
        fd_ctx.set_state(scn.initial_state())
        act = [fd_ctx.ipc_step(params(m))["n_active"] for _ in range(steps)]
        S = fd_ctx.state()
        return float(((S["position"] - tgt_p) ** 2).sum() + ((S["orientation"] - tgt_q) ** 2).sum()), act

    checks = []
    h = 1e-4 * mu
    (lp, ap), (lm, am) = loss(sc, mu + h), loss(sc, mu - h)
    assert ap == branch and am == branch
    checks.append((g["friction"], (lp - lm) / (2 * h)))
    for b, k in ((1, 0), (2, 2), (3, 0)):
        vp, vm = sc.velocity.copy(), sc.velocity.copy()
        vp[b, k] += 1e-4
        vm[b, k] -= 1e-4
        (lp, ap), (lm, am) = (loss(adjoint.with_parameters(sc, velocity=vp), mu),
                              loss(adjoint.with_parameters(sc, velocity=vm), mu))
        if ap == branch and am == branch:
            checks.append((g["velocity"][b, k], (lp - lm) / 2e-4))
    a = np.array(checks)
    assert np.abs(a[:, 0] - a[:, 1]).max() <= 1e-3 * np.abs(a[:, 1]).max(), a


def test_autograd_function_passes_the_adjoint_through():
    # torch.autograd over the rollout function: the gradients of velocity,
    # mass, joint stiffness and friction coefficient equal IpcRollout's
    import torch
    sc = scenes.diff_ipc_scene(n_spheres=4)
    P = abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-9, newton_max_iters=100, ls_max_iters=40,
                       mu=0.4, friction_eps=1e-5, friction_iters=1)
    fn = adjoint.make_rollout_function()
    v0 = torch.tensor(sc.velocity, requires_grad=True)
    m = torch.tensor(sc.mass, requires_grad=True)
    mu = torch.tensor(sc.joint_stiffness, requires_grad=True)
    fr = torch.tensor(0.4, dtype=torch.float64, requires_grad=True)
    out = fn.apply(v0, m, mu, sc, P, 8, 3, fr)
    tgt = out.detach() + 0.01
    ((out - tgt) ** 2).sum().backward()
    r = adjoint.IpcRollout(sc, P, checkpoint_every=3)
    T = r.forward(8)
    o = np.concatenate([T["position"], T["orientation"]], 1)
    g = r.backward(2 * (o[:, :3] - tgt.numpy()[:, :3]), 2 * (o[:, 3:] - tgt.numpy()[:, 3:]))
    assert np.allclose(v0.grad.numpy(), g["velocity"], rtol=1e-12, atol=0)
    assert np.allclose(m.grad.numpy(), g["mass"], rtol=1e-12, atol=0)
    assert np.allclose(mu.grad.numpy(), g["joint_stiffness"], rtol=1e-12, atol=0)
    assert float(fr.grad) == pytest.approx(g["friction"], rel=1e-12)
