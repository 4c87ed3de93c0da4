"""The trajectory fixtures of the measured configurations against the CPU
oracle (no GPU): a fixture must be the oracle's run of its seeded scene, so
a change to the oracle or to a scene generator shows up here before the GPU
tests compare the device with it.  Short prefixes keep this to seconds: the
sphere bowl's first checkpoint (20 steps), the hopper's first two steps'
counts and fingerprints, and the first 10 steps of a few batched scenes.
"""
import os

import numpy as np

from nexdynipc_b200 import scenes
from oracle import refcpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fingerprint(st):
    return (float(st["position"].sum()),
            float((st["orientation"] * np.array([1.0, 2.0, 3.0, 4.0])).sum()))


def test_sphere_bowl_fixture_is_the_oracle_run():
    ref = np.load(os.path.join(GOLDEN, "traj_sphere_bowl.npz"))
    assert list(ref["checkpoint_steps"]) == list(range(20, 201, 20))
    ow = refcpu.OracleWorld(scenes.sphere_bowl(), threads=os.cpu_count() or 1)
    for s in range(20):
        ow.step()
        d = ow.diagnostics()
        assert d["n_contacts"] == ref["n_contacts"][s] and d["kappa"] == ref["kappa"][s]
        assert fingerprint(ow.state()) == tuple(ref["fp"][s])
    st = ow.state()
    assert np.array_equal(st["position"], ref["position"][0])
    assert np.array_equal(st["orientation"], ref["orientation"][0])


def test_hopper_fixture_first_steps():
    ref = np.load(os.path.join(GOLDEN, "traj_hopper_chains.npz"))
    sc = scenes.hopper_chains()
    assert ref["position"].shape == (5, sc.n_bodies, 3)
    ow = refcpu.OracleWorld(sc, threads=os.cpu_count() or 1)
    for s in range(2):
        ow.step()
        d = ow.diagnostics()
        for k in ("n_contacts", "alm_iterations", "newton_iterations"):
            assert d[k] == ref[k][s], (k, s)
        assert fingerprint(ow.state()) == tuple(ref["fp"][s])


def test_batched_fixture_first_steps():
    ref = np.load(os.path.join(GOLDEN, "traj_batched.npz"))
    scs = scenes.batched_scenes()
    assert ref["fp"].shape == (256, 10, 2) and ref["diag"].shape == (256, 100, 3)
    for i in (0, 1, 77, 255):
        ow = refcpu.OracleWorld(scs[i])
        for s in range(10):
            ow.step()
            d = ow.diagnostics()
            assert [d["n_contacts"], d["alm_iterations"], d["newton_iterations"]] == list(ref["diag"][i, s])
        assert fingerprint(ow.state()) == tuple(ref["fp"][i, 0])


def test_ipc_sphere_bowl_fixture_first_step():
    from nexdynipc_b200 import abi
    ref = np.load(os.path.join(GOLDEN, "traj_ipc_sphere_bowl.npz"))
    assert ref["position"].shape == (40, 65, 3)
    ow = refcpu.OracleWorld(scenes.sphere_bowl())
    st = ow.ipc_step(abi.ipc_params(**scenes.ipc_step_settings()))
    for k in ("newton_iterations", "converged", "line_search_failed", "n_active", "n_pairs"):
        assert st[k] == ref[k][0], k
    s = ow.state()
    assert np.array_equal(s["position"], ref["position"][0])
    assert np.array_equal(s["orientation"], ref["orientation"][0])
