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
