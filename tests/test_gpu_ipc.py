"""GPU parity of the primitive-level contact model (full IPC) against its
oracle, through the C ABI (nxd_ipc_candidates / nxd_ipc_barrier /
nxd_ipc_max_step).

Candidate sets must be identical (sorted pair lists).  Energies, gradients
and Hessian blocks are compared within 1e-10 relative; both sides run the
same per-pair arithmetic without FMA contraction and sum in the same fixed
orders, so they agree bit for bit, which the tests report.  The CCD bound
must not exceed the oracle's by more than 1e-12 (it equals it), and it
follows the rigid rotation arcs of the iterates.
"""
import numpy as np
import pytest

from nexdynipc_b200 import scenes
from oracle import refcpu

pytestmark = pytest.mark.gpu


def runtime():
    from nexdynipc_b200 import runtime as rt
    return rt


def scene_x(sc, seed, jitter):
    rng = np.random.default_rng(seed)
    x = np.zeros(6 * sc.n_bodies)
    for i in range(sc.n_bodies):
        x[6 * i:6 * i + 3] = sc.position[i] + rng.normal(0, jitter, 3)
        x[6 * i + 3:6 * i + 6] = rng.normal(0, jitter, 3)
    return x


SCENES = {
    "cube_stack": (lambda: scenes.cube_stack(), 1e-4),
    "sphere_bowl": (lambda: scenes.sphere_bowl(n_spheres=24), 5e-3),
    "hopper_small": (lambda: scenes.hopper_chains(n_hulls=192, n_chains=6), 1e-3),
}


def bsr_dense(n, rp, ci, vv):
    H = np.zeros((6 * n, 6 * n))
    for r in range(n):
        for k in range(rp[r], rp[r + 1]):
            H[6 * r:6 * r + 6, 6 * ci[k]:6 * ci[k] + 6] = vv[k]
    return H


@pytest.mark.parametrize("name", list(SCENES))
def test_ipc_candidates_identical(name):
    make, jitter = SCENES[name]
    sc = make()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, 1, jitter)
    dhat = sc.settings.dhat
    for infl in (0.0, dhat, 0.02):
        gpt, gee = ctx.ipc_candidates(x, None, infl)
        opt, oee = ow.ipc_candidates(x, None, infl)
        assert np.array_equal(gpt, opt), (infl, len(gpt), len(opt))
        assert np.array_equal(gee, oee), (infl, len(gee), len(oee))
    # current poses, and swept boxes over a step
    assert all(np.array_equal(a, b) for a, b in zip(ctx.ipc_candidates(None, None, dhat), ow.ipc_candidates(None, None, dhat)))
    dx = np.random.default_rng(2).normal(0, 2e-3, x.shape)
    for a, b in zip(ctx.ipc_candidates(x, dx, 0.0), ow.ipc_candidates(x, dx, 0.0)):
        assert np.array_equal(a, b)


def long_slice_scene():
    """A 2562-vertex icosphere (7680 edges) resting on a 12-triangle box: the
    box's edges are queries whose hits cover the sphere's edges."""
    sb = scenes.SceneBuilder("long_slices")
    gv, gf = scenes.box_mesh(0.3, 0.05, 0.3)
    g = sb.add_body(gv, gf, (0.0, -0.05, 0.0))
    sb.fix(g)
    iv, if_ = scenes.icosphere(4)
    sb.add_body(iv * 0.1, if_, (0.0, 0.1005, 0.0))
    return sb.build(scenes._settings(1e-3, 0.0), dt=1e-2, steps=1)


def test_ipc_candidates_long_slices():
    """Candidate lists whose longest per-query slice takes each sort: at
    inflation 0.02 the longest edge slice has 800 pairs (past the per-lane
    insertion sort, inside a warp's shared row); at 0.5 the slices reach
    5120 and 7680 pairs (the radix sort of packed keys)."""
    sc = long_slice_scene()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, 1, 1e-5)
    for infl, longest in ((0.02, 800), (0.5, 7680)):
        gpt, gee = ctx.ipc_candidates(x, None, infl)
        opt, oee = ow.ipc_candidates(x, None, infl)
        assert max(np.bincount(a[:, 0]).max() for a in (opt, oee)) == longest
        assert np.array_equal(gpt, opt), (infl, len(gpt), len(opt))
        assert np.array_equal(gee, oee), (infl, len(gee), len(oee))


@pytest.mark.parametrize("name", list(SCENES))
def test_ipc_barrier_matches_oracle(name):
    make, jitter = SCENES[name]
    sc = make()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, 3, jitter * 0.5)
    dhat = max(sc.settings.dhat, 2e-3)
    kappa = 1e5
    eg, gg, (rp, ci, vv), npg, nag = ctx.ipc_barrier(x, dhat, kappa)
    eo, go, Ho, npo, nao = ow.ipc_barrier(x, dhat, kappa)
    assert (npg, nag) == (npo, nao)
    assert nag > 0, "the state has no active pair"
    assert abs(eg - eo) <= 1e-10 * abs(eo)
    assert np.abs(gg - go).max() <= 1e-10 * np.abs(go).max()
    Hg = bsr_dense(sc.n_bodies, rp, ci, vv)
    assert np.abs(Hg - Ho).max() <= 1e-10 * np.abs(Ho).max()
    assert np.count_nonzero(np.abs(Ho).reshape(sc.n_bodies, 6, sc.n_bodies, 6).sum((1, 3))) <= len(ci)
    print(f"{name}: {npg} pairs, {nag} active; energy/gradient/Hessian bit-equal:",
          eg == eo, np.array_equal(gg, go), np.array_equal(Hg, Ho))


@pytest.mark.parametrize("name", list(SCENES))
def test_ipc_max_step_matches_oracle(name):
    make, jitter = SCENES[name]
    sc = make()
    ctx = runtime().Context(sc)
    ow = refcpu.OracleWorld(sc)
    x = scene_x(sc, 4, jitter * 0.5)
    rng = np.random.default_rng(5)
    dx = np.zeros_like(x)
    for i in range(sc.n_bodies):   # bodies pushed together, small rotations
        dx[6 * i:6 * i + 3] = -0.05 * (x[6 * i:6 * i + 3] - x[0:3]) + rng.normal(0, 0.01, 3)
        dx[6 * i + 3:6 * i + 6] = rng.normal(0, 0.02, 3)
    ag, ng = ctx.ipc_max_step(x, dx, 0.1)
    ao, no = ow.ipc_max_step(x, dx, 0.1)
    assert ng == no
    assert 0.0 <= ag <= 1.0
    assert ag <= ao + 1e-12
    assert ag == ao


def test_ipc_max_step_follows_the_rotation_arc():
    # the oracle's arc case (tests/test_ipc_oracle.py): a cube turned by 90
    # degrees whose corners swing below the ground half-way; the device bound
    # equals the oracle's bit for bit and stops before the arc's contact
    sc = scenes.ipc_drop(n_cubes=1)
    st = sc.initial_state()
    st["orientation"][1] = [1.0, 0.0, 0.0, 0.0]
    st["position"][1] = [0.0, 0.125, 0.0]
    st["velocity"][1] = 0.0
    st["angular_velocity"][1] = 0.0
    ctx = runtime().Context(sc)
    ctx.set_state(st)
    ow = refcpu.OracleWorld(sc)
    ow.set_state(st)
    x = np.zeros(6 * sc.n_bodies)
    x.reshape(-1, 6)[:, :3] = st["position"]
    dx = np.zeros_like(x)
    dx[6 + 5] = np.pi / 2
    ag, ng = ctx.ipc_max_step(x, dx, 0.1)
    ao, no = ow.ipc_max_step(x, dx, 0.1)
    assert ng == no and ag == ao and 0.1 < ag < 0.19, (ag, ao)
