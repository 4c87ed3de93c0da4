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
