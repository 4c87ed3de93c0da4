"""GPU trajectory parity at the measured configurations' full sizes.

The device steps each configuration from its seeded scene through its whole
run, through the C ABI, and is compared with the CPU oracle's run of the
same scene stored in tests/golden/traj_*.npz (make_trajectory_goldens.py):

* the 1024-hull hopper with 32 hinge chains (1313 bodies), 100 steps;
* 64 icospheres (642 V) falling into the bowl, 200 steps;
* the 256 uneven batched scenes, 100 steps, as one batch;
* the 64-sphere bowl stepped by the full-IPC step (nxd_ipc_step), 40 steps
  against the oracle's nxo_ipc_step (traj_ipc_sphere_bowl.npz), and 20 steps
  with lagged friction mu 0.3 (traj_ipc_sphere_bowl_friction.npz).

Every step: adaptive stiffness, contact count and ALM / Newton iteration
counts equal, and the position / orientation fingerprints within the
trajectory tolerance summed over bodies.  At the checkpoints: every body
within 1e-6 m and 1e-6 rad.  Both sides round every operation the same way,
so the runs are expected to agree bit for bit; the tests assert the
tolerance and report the worst difference.
"""
import os

import numpy as np
import pytest

from nexdynipc_b200 import scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_P = 1e-6     # m
TOL_R = 1e-6     # rad


def quat_angle(qa, qb):
    """Rotation angle of qa^-1 qb per body: 2 atan2(|vec|, |w|), accurate near
    zero (2 acos(|qa.qb|) bottoms out near 3e-8 rad in FP64)."""
    w = np.einsum("ij,ij->i", qa, qb)
    va, vb = qa[:, 1:], qb[:, 1:]
    vec = qa[:, :1] * vb - qb[:, :1] * va - np.cross(va, vb)
    return 2 * np.arctan2(np.linalg.norm(vec, axis=1), np.abs(w))


def fingerprint(st):
    return (float(st["position"].sum()),
            float((st["orientation"] * np.array([1.0, 2.0, 3.0, 4.0])).sum()))


def run_against_fixture(sc, name):
    from nexdynipc_b200 import runtime
    ref = np.load(os.path.join(GOLDEN, f"traj_{name}.npz"))
    ctx = runtime.Context(sc)
    n = sc.n_bodies
    ck = list(ref["checkpoint_steps"])
    worst_p = worst_r = 0.0
    for s in range(sc.steps):
        ctx.step()
        d = ctx.diagnostics()
        assert d["status"] == 0, (s, d["status"])
        assert d["kappa"] == ref["kappa"][s], s
        assert d["n_contacts"] == ref["n_contacts"][s], s
        assert d["alm_iterations"] == ref["alm_iterations"][s], s
        assert d["newton_iterations"] == ref["newton_iterations"][s], s
        st = ctx.state()
        fp = fingerprint(st)
        assert abs(fp[0] - ref["fp"][s, 0]) <= n * TOL_P, s
        assert abs(fp[1] - ref["fp"][s, 1]) <= 10 * n * TOL_R, s
        if (s + 1) in ck:
            c = ck.index(s + 1)
            worst_p = max(worst_p, float(np.abs(st["position"] - ref["position"][c]).max()))
            worst_r = max(worst_r, float(quat_angle(st["orientation"], ref["orientation"][c]).max()))
    lam, mu = ctx.joint_state()
    ctx.close()
    return worst_p, worst_r, lam, mu, ref


def test_hopper_chains_full_run():
    # the configuration bench.py times: 1313 bodies, 100 steps
    wp, wr, lam, mu, ref = run_against_fixture(scenes.hopper_chains(), "hopper_chains")
    print(f"hopper_chains 100 steps: max |dp| {wp:.3e} m, max rotation {wr:.3e} rad")
    assert wp <= TOL_P and wr <= TOL_R, (wp, wr)
    assert np.array_equal(mu, ref["joint_mu"])
    assert np.abs(lam - ref["joint_lambda"]).max() <= 1e-6 * max(1.0, np.abs(ref["joint_lambda"]).max())


def test_sphere_bowl_full_run():
    wp, wr, _, _, _ = run_against_fixture(scenes.sphere_bowl(), "sphere_bowl")
    print(f"sphere_bowl 200 steps: max |dp| {wp:.3e} m, max rotation {wr:.3e} rad")
    assert wp <= TOL_P and wr <= TOL_R, (wp, wr)


def test_batched_256_scenes_full_run():
    from nexdynipc_b200 import runtime
    ref = np.load(os.path.join(GOLDEN, "traj_batched.npz"))
    scs = scenes.batched_scenes()
    off = ref["body_offset"]
    assert len(scs) == 256 and off[-1] == sum(s.n_bodies for s in scs)
    b = runtime.Batch(scs)
    worst_p = worst_r = 0.0
    for s in range(100):
        b.step()
        for i in range(len(scs)):
            d = b.diagnostics(i)
            assert d["status"] == 0, (i, s)
            assert [d["n_contacts"], d["alm_iterations"], d["newton_iterations"]] == list(ref["diag"][i, s]), (i, s)
        if (s + 1) % 10 == 0:
            for i, sc in enumerate(scs):
                st = b.state(i)
                fp = fingerprint(st)
                r = ref["fp"][i, (s + 1) // 10 - 1]
                assert abs(fp[0] - r[0]) <= sc.n_bodies * TOL_P, (i, s)
                assert abs(fp[1] - r[1]) <= 10 * sc.n_bodies * TOL_R, (i, s)
                if s + 1 in (50, 100):
                    want = ref["state_50" if s + 1 == 50 else "state_100"][off[i]:off[i + 1]]
                    worst_p = max(worst_p, float(np.abs(st["position"] - want[:, :3]).max()))
                    worst_r = max(worst_r, float(quat_angle(st["orientation"], want[:, 3:]).max()))
    b.close()
    print(f"batched 256 scenes x 100 steps: max |dp| {worst_p:.3e} m, max rotation {worst_r:.3e} rad")
    assert worst_p <= TOL_P and worst_r <= TOL_R, (worst_p, worst_r)


def run_ipc_against_fixture(name, mu):
    from nexdynipc_b200 import abi, runtime
    ref = np.load(os.path.join(GOLDEN, f"traj_{name}.npz"))
    sc = scenes.sphere_bowl()
    ctx = runtime.Context(sc)
    p = abi.ipc_params(**scenes.ipc_step_settings(mu=mu))
    worst_p = worst_r = 0.0
    keys = [k for k in ("newton_iterations", "converged", "line_search_failed", "n_active", "n_pairs", "n_friction")
            if k in ref.files]
    for s in range(ref["position"].shape[0]):
        st = ctx.ipc_step(p)     # raises on a non-zero status
        for k in keys:
            assert st[k] == ref[k][s], (s, k, st[k], ref[k][s])
        S = ctx.state()
        worst_p = max(worst_p, float(np.abs(S["position"] - ref["position"][s]).max()))
        worst_r = max(worst_r, float(quat_angle(S["orientation"], ref["orientation"][s]).max()))
        assert worst_p <= TOL_P and worst_r <= TOL_R, (s, worst_p, worst_r)
    ctx.close()
    return ref["position"].shape[0], worst_p, worst_r


def test_sphere_bowl_full_ipc_steps():
    # the primitive-pair model on the 64-sphere configuration: every step's
    # Newton count, flags and active / candidate pair counts equal, every
    # body within 1e-6 m and 1e-6 rad of the oracle's step at every step
    n, wp, wr = run_ipc_against_fixture("ipc_sphere_bowl", 0.0)
    print(f"sphere_bowl full IPC {n} steps: max |dp| {wp:.3e} m, max rotation {wr:.3e} rad")


def test_sphere_bowl_full_ipc_friction_steps():
    # the same with the configuration's mu 0.3 as lagged friction (two passes)
    n, wp, wr = run_ipc_against_fixture("ipc_sphere_bowl_friction", 0.3)
    print(f"sphere_bowl full IPC + friction {n} steps: max |dp| {wp:.3e} m, max rotation {wr:.3e} rad")
