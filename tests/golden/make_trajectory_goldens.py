"""Writes the trajectory fixtures of the measured configurations.

Each fixture is the CPU oracle's run of one configuration from its seeded
scene (``nexdynipc_b200.scenes``), with the oracle's pruned scene minimum
distance (exact below 1e-6, so the adaptive-stiffness decisions equal the
literal loop's) on all host threads:

* ``traj_hopper_chains.npz`` -- 1024 hulls + 32 hinge chains (1313 bodies),
  100 steps of dt 5e-3;
* ``traj_sphere_bowl.npz``   -- 64 icospheres (642 V) in the bowl, 200 steps;
* ``traj_batched.npz``       -- the 256 uneven scenes, 100 steps each;
* ``traj_ipc_sphere_bowl.npz`` -- the same 64-sphere bowl stepped by the
  full-IPC step (primitive-pair barrier, additive-CCD line search; the
  oracle's nxo_ipc_step with scenes.ipc_step_settings()), its first 40 steps;
* ``traj_ipc_sphere_bowl_friction.npz`` -- the same with the configuration's
  mu 0.3 as lagged friction (scenes.ipc_step_settings(mu=0.3)), 20 steps.

Stored per fixture: positions and orientations at the checkpoint steps, and
for every step the adaptive stiffness kappa, the contact count, the ALM and
Newton iteration counts and a position / orientation fingerprint (sums over
bodies), so a device run can be compared with the oracle at every step
without storing every state.  The batched fixture keeps the states of steps
50 and 100 and the per-scene fingerprints every 10 steps.

The full-IPC fixture stores, for every step, the Newton iteration count, the
convergence and line-search flags, the active and candidate pair counts and
the full body state (positions, orientations).

Usage: python tests/golden/make_trajectory_goldens.py [hopper|bowl|batched|ipc_bowl|ipc_bowl_friction ...]
(about 8 minutes for the hopper on 8 threads, a few minutes for the others).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from nexdynipc_b200 import scenes  # noqa: E402

DIAG_KEYS = ("kappa", "n_contacts", "alm_iterations", "newton_iterations")


def fingerprint(st):
    """(sum of positions, sum of orientations weighted 1..4) over bodies."""
    return (float(st["position"].sum()),
            float((st["orientation"] * np.array([1.0, 2.0, 3.0, 4.0])).sum()))


def run_single(sc, every, threads):
    from oracle import refcpu
    ow = refcpu.OracleWorld(sc, threads=threads)
    n = sc.steps
    out = {k: np.zeros(n) for k in ("kappa",)}
    for k in ("n_contacts", "alm_iterations", "newton_iterations"):
        out[k] = np.zeros(n, np.int32)
    out["fp"] = np.zeros((n, 2))
    ck_steps = [s for s in range(every, n + 1, every)]
    pos, quat = [], []
    t0 = time.time()
    for s in range(n):
        ow.step()
        d = ow.diagnostics()
        for k in DIAG_KEYS:
            out[k][s] = d[k]
        st = ow.state()
        out["fp"][s] = fingerprint(st)
        if (s + 1) in ck_steps:
            pos.append(st["position"])
            quat.append(st["orientation"])
        if (s + 1) % 10 == 0:
            print(f"  {sc.name}: step {s + 1}/{n}, {time.time() - t0:.0f} s", flush=True)
    out["checkpoint_steps"] = np.array(ck_steps, np.int32)
    out["position"] = np.stack(pos)
    out["orientation"] = np.stack(quat)
    lam, mu = ow.joint_state()
    out["joint_lambda"], out["joint_mu"] = lam, mu
    return out


def _batched_one(si):
    from oracle import refcpu
    sc = _SCENES[si]
    ow = refcpu.OracleWorld(sc, threads=1)
    fps, states, diag = [], [], []
    for s in range(sc.steps):
        ow.step()
        d = ow.diagnostics()
        diag.append([d["n_contacts"], d["alm_iterations"], d["newton_iterations"]])
        if (s + 1) % 10 == 0:
            st = ow.state()
            fps.append(fingerprint(st))
            if (s + 1) in (50, 100):
                states.append(np.concatenate([st["position"], st["orientation"]], 1))
    return si, np.array(fps), states, np.array(diag, np.int32)


_SCENES = None


def _init_batched():
    global _SCENES
    _SCENES = scenes.batched_scenes()


def make_batched(path):
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count(), initializer=_init_batched) as pool:
        res = sorted(pool.map(_batched_one, range(256)), key=lambda r: r[0])
    scs = scenes.batched_scenes()
    off = np.zeros(len(scs) + 1, np.int64)
    off[1:] = np.cumsum([s.n_bodies for s in scs])
    s50 = np.concatenate([r[2][0] for r in res])
    s100 = np.concatenate([r[2][1] for r in res])
    np.savez_compressed(path, body_offset=off, fp=np.stack([r[1] for r in res]),
                        diag=np.stack([r[3] for r in res]),
                        state_50=s50, state_100=s100)


IPC_STAT_KEYS = ("newton_iterations", "converged", "line_search_failed", "n_active", "n_pairs", "n_friction")


def run_ipc(sc, steps, mu=0.0):
    from nexdynipc_b200 import abi
    from oracle import refcpu
    ow = refcpu.OracleWorld(sc)
    p = abi.ipc_params(**scenes.ipc_step_settings(mu=mu))
    out = {k: np.zeros(steps, np.int64) for k in IPC_STAT_KEYS}
    pos, quat = [], []
    t0 = time.time()
    for s in range(steps):
        st = ow.ipc_step(p)
        assert st["status"] == 0, (s, st)
        for k in IPC_STAT_KEYS:
            out[k][s] = st[k]
        S = ow.state()
        pos.append(S["position"])
        quat.append(S["orientation"])
        if (s + 1) % 10 == 0:
            print(f"  {sc.name} (full IPC): step {s + 1}/{steps}, {time.time() - t0:.0f} s", flush=True)
    out["position"] = np.stack(pos)
    out["orientation"] = np.stack(quat)
    return out


def main(which):
    if "hopper" in which:
        t = time.time()
        out = run_single(scenes.hopper_chains(), 20, os.cpu_count())
        np.savez_compressed(os.path.join(HERE, "traj_hopper_chains.npz"), **out)
        print(f"hopper: {time.time() - t:.0f} s")
    if "bowl" in which:
        t = time.time()
        out = run_single(scenes.sphere_bowl(), 20, os.cpu_count())
        np.savez_compressed(os.path.join(HERE, "traj_sphere_bowl.npz"), **out)
        print(f"bowl: {time.time() - t:.0f} s")
    if "ipc_bowl" in which:
        t = time.time()
        out = run_ipc(scenes.sphere_bowl(), 40)
        np.savez_compressed(os.path.join(HERE, "traj_ipc_sphere_bowl.npz"), **out)
        print(f"ipc_bowl: {time.time() - t:.0f} s")
    if "ipc_bowl_friction" in which:
        t = time.time()
        out = run_ipc(scenes.sphere_bowl(), 20, mu=0.3)
        np.savez_compressed(os.path.join(HERE, "traj_ipc_sphere_bowl_friction.npz"), **out)
        print(f"ipc_bowl_friction: {time.time() - t:.0f} s")
    if "batched" in which:
        t = time.time()
        make_batched(os.path.join(HERE, "traj_batched.npz"))
        print(f"batched: {time.time() - t:.0f} s")


if __name__ == "__main__":
    main(sys.argv[1:] or ["hopper", "bowl", "batched"])
