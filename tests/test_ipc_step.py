"""Full-IPC time step (nxd_ipc_step; oracle nxo_ipc_step): the primitive-pair
barrier, CCD-bounded line search and block LDL^T solve inside one Newton
step.  The CPU tests check the oracle's step against the guarantees of the
method (no surface crossed, Newton converged, bodies at rest in contact);
the GPU test checks the device step against the oracle's."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu

PARAMS = dict(dhat=1e-3, kappa=1e11, eta=0.1, newton_tol=1e-6, newton_max_iters=50, ls_max_iters=30)


def quat_rot(q, v):
    w, u = q[0], q[1:]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def world_vertices(sc, st, b):
    v = sc.vertices[sc.vertex_offset[b]:sc.vertex_offset[b + 1]]
    return np.array([st["position"][b] + quat_rot(st["orientation"][b], p) for p in v])


def test_oracle_ipc_step_keeps_bodies_apart_and_converges():
    sc = scenes.ipc_drop(n_cubes=2)
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**PARAMS)
    for k in range(60):
        st = ow.ipc_step(p)
        assert st["status"] == 0 and st["line_search_failed"] == 0
        assert st["converged"] == 1, (k, st)
        s = ow.state()
        # the ground's top face is y = 0: no cube vertex below it
        for b in (1, 2):
            assert world_vertices(sc, s, b)[:, 1].min() > 0.0, (k, b)
    s = ow.state()
    # both at rest: the lower cube on the ground within dhat, the upper on it
    assert np.abs(s["velocity"][1:]).max() < 0.05
    assert world_vertices(sc, s, 1)[:, 1].min() < 1e-3
    assert s["position"][2, 1] > s["position"][1, 1] + 0.15


def test_oracle_ipc_step_barrier_strength_matters():
    # a barrier too weak to carry the cube's weight: once the cube reaches
    # the ground every Newton step is cut by the CCD bound and Newton runs
    # out of iterations instead of converging
    sc = scenes.ipc_drop(n_cubes=1)
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**dict(PARAMS, kappa=1e5, newton_max_iters=8))
    capped = 0
    for _ in range(20):
        st = ow.ipc_step(p)
        if st["last_alpha_max"] < 1.0 and st["converged"] == 0 and st["newton_iterations"] == 8:
            capped += 1
    assert capped >= 3


@pytest.mark.gpu
def test_device_ipc_step_matches_oracle():
    from nexdynipc_b200 import runtime
    sc = scenes.ipc_drop(n_cubes=3)
    ctx = runtime.Context(sc)
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**PARAMS)
    worst = 0.0
    for k in range(40):
        sg = ctx.ipc_step(p)
        so = ow.ipc_step(p)
        assert sg["newton_iterations"] == so["newton_iterations"], (k, sg, so)
        assert sg["n_active"] == so["n_active"] and sg["converged"] == so["converged"]
        a, b = ctx.state(), ow.state()
        worst = max(worst, float(np.abs(a["position"] - b["position"]).max()))
        assert worst <= 1e-6, (k, worst)
    assert ctx.diagnostics()["status"] == 0


@pytest.mark.gpu
def test_device_ipc_step_trial_overflow_path_matches_oracle(monkeypatch):
    # every line-search trial's candidate lists forced over their capacity
    # (NXD_IPC_TRIAL_CAP=0): each trial takes the two-wait fallback, and the
    # step must still equal the oracle's bit for bit
    from nexdynipc_b200 import runtime
    monkeypatch.setenv("NXD_IPC_TRIAL_CAP", "0")
    sc = scenes.ipc_drop(n_cubes=3)
    ctx = runtime.Context(sc)
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**PARAMS)
    trials = 0
    for k in range(30):
        sg = ctx.ipc_step(p)
        so = ow.ipc_step(p)
        assert sg["newton_iterations"] == so["newton_iterations"], (k, sg, so)
        assert sg["n_active"] == so["n_active"] and sg["converged"] == so["converged"]
        a, b = ctx.state(), ow.state()
        assert np.array_equal(a["position"], b["position"]), k
        assert np.array_equal(a["orientation"], b["orientation"]), k
        trials += sg["newton_iterations"]
    assert trials > 0
    assert ctx.diagnostics()["status"] == 0


@pytest.mark.gpu
def test_device_ipc_step_with_pcg_tracks_the_direct_solve():
    # the same step with block-Jacobi PCG (tolerance 1e-13) for the Newton
    # systems stays on the oracle's direct-solve trajectory
    from nexdynipc_b200 import runtime
    sc = scenes.ipc_drop(n_cubes=3)
    ctx = runtime.Context(sc)
    ow = refcpu.OracleWorld(sc)
    pg = abi.ipc_params(**PARAMS, linear_solver=abi.IPC_SOLVER_PCG, pcg_max_iter=500, pcg_tol=1e-13)
    po = abi.ipc_params(**PARAMS)
    used = 0
    for k in range(30):
        sg = ctx.ipc_step(pg)
        so = ow.ipc_step(po)
        used += sg["pcg_iterations"]
        assert sg["solve_failed"] == 0
        d = float(np.abs(ctx.state()["position"] - ow.state()["position"]).max())
        assert d <= 1e-6, (k, d)
    assert used > 0


def settled_cube(mu_steps=30):
    """One 0.2 m cube settled on the ground (30 frictionless steps), then
    given 1 m/s along x."""
    sc = scenes.ipc_drop(n_cubes=1)
    ow = refcpu.OracleWorld(sc)
    p0 = abi.ipc_params(**scenes.ipc_step_settings())
    for _ in range(mu_steps):
        ow.ipc_step(p0)
    S = ow.state()
    S["velocity"][1] = [1.0, 0.0, 0.0]
    S["angular_velocity"][1] = 0.0
    return sc, ow, S


def test_oracle_friction_derivatives():
    # the friction of the pairs frozen at x_lag: gradient = central
    # differences of the energy; the translation blocks of the Gauss-Newton
    # Hessian = central differences of the gradient (the map is linear in
    # translations); the Hessian symmetric and PSD
    sc = scenes.ipc_drop(n_cubes=2)
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**scenes.ipc_step_settings())
    for _ in range(30):
        ow.ipc_step(p)
    n = 6 * sc.n_bodies
    xl = np.zeros(n)
    xl.reshape(-1, 6)[:, :3] = ow.state()["position"]
    x = xl + np.random.default_rng(0).normal(size=n) * 2e-4
    args = (1e-3, 1e11, 0.5, 1e-5)
    e, g, H, nf = ow.ipc_friction(xl, x, *args)
    assert nf > 0 and e > 0.0
    h = 1e-7
    gf, Hf = np.zeros(n), np.zeros((n, n))
    for i in range(n):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        ep, gp, _, _ = ow.ipc_friction(xl, xp, *args, hessian=False)
        em, gm, _, _ = ow.ipc_friction(xl, xm, *args, hessian=False)
        gf[i] = (ep - em) / (2 * h)
        Hf[:, i] = (gp - gm) / (2 * h)
    assert np.abs(g - gf).max() <= 1e-6 * np.abs(g).max()
    tr = np.array([i for i in range(n) if i % 6 < 3])
    assert np.abs(H[np.ix_(tr, tr)] - Hf[np.ix_(tr, tr)]).max() <= 1e-5 * np.abs(H).max()
    assert np.abs(H - H.T).max() <= 1e-12 * np.abs(H).max()
    assert np.linalg.eigvalsh(H).min() >= -1e-12 * np.abs(H).max()


def test_oracle_friction_decelerates_and_sticks():
    # a cube sliding at 1 m/s: frictionless it keeps its speed; with mu it
    # slows by mu g per second (Coulomb) and then stays at rest (static
    # friction of the smoothed potential, eps 1e-5 m)
    for mu in (0.0, 0.2, 0.5):
        sc, ow, S = settled_cube()
        ow.set_state(S)
        p = abi.ipc_params(**dict(scenes.ipc_step_settings(), mu=mu, friction_eps=1e-5, friction_iters=2))
        vx = []
        for k in range(40):
            st = ow.ipc_step(p)
            assert st["status"] == 0 and st["converged"] == 1 and st["line_search_failed"] == 0, (mu, k, st)
            vx.append(ow.state()["velocity"][1][0])
        if mu == 0.0:
            assert st["n_friction"] == 0 and abs(vx[-1] - 1.0) < 5e-3
        elif mu == 0.2:
            decel = (vx[5] - vx[35]) / (30 * sc.dt)
            assert abs(decel - mu * 9.81) < 0.02 * mu * 9.81, decel
        else:
            assert st["n_friction"] > 0
            assert max(abs(v) for v in vx[25:]) < 2e-3, vx


@pytest.mark.gpu
def test_device_ipc_step_friction_matches_oracle():
    # lagged friction over two passes, on a sliding cube and on a dropped
    # three-cube stack: every step's counts equal the oracle's and the
    # positions agree (both round every operation the same way)
    from nexdynipc_b200 import runtime
    cases = []
    sc, ow, S = settled_cube()
    ow.set_state(S)
    ctx = runtime.Context(sc)
    ctx.set_state(S)
    cases.append((ctx, ow, 0.5))
    sc3 = scenes.ipc_drop(n_cubes=3)
    cases.append((runtime.Context(sc3), refcpu.OracleWorld(sc3), 0.3))
    for ctx, ow, mu in cases:
        p = abi.ipc_params(**dict(scenes.ipc_step_settings(), mu=mu, friction_eps=1e-5, friction_iters=2))
        worst = 0.0
        for k in range(40):
            sg = ctx.ipc_step(p)
            so = ow.ipc_step(p)
            for key in ("newton_iterations", "converged", "line_search_failed", "n_active", "n_pairs", "n_friction"):
                assert sg[key] == so[key], (mu, k, key, sg, so)
            a, b = ctx.state(), ow.state()
            worst = max(worst, float(np.abs(a["position"] - b["position"]).max()))
            assert worst <= 1e-9, (mu, k, worst)
        ctx.close()
