"""LinearSolver on a caller's block matrix (nxd_linear_solve) and the fused
SimulationProblem call (nxd_eval_all): the oracle against the dense solve,
the device against the oracle."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu


def random_block_system(n=9, seed=0, dup=True):
    """A symmetric positive definite 6x6-block matrix on a chain plus a star,
    in BSR with both triangles stored and some blocks split into two
    duplicates (summed in storage order)."""
    rng = np.random.default_rng(seed)
    edges = [(i, i + 1) for i in range(n - 1)] + [e for e in ((0, n - 1), (2, 6)) if e[1] < n and e[1] - e[0] > 1]
    dense = np.zeros((6 * n, 6 * n))
    blocks = {i: [] for i in range(n)}
    for a, b in edges:
        B = rng.normal(size=(6, 6)) * 0.3
        dense[6 * a:6 * a + 6, 6 * b:6 * b + 6] += B
        dense[6 * b:6 * b + 6, 6 * a:6 * a + 6] += B.T
        if dup and (a + b) % 3 == 0:
            h = rng.normal(size=(6, 6)) * 0.1
            blocks[a] += [(b, B - h), (b, h)]
        else:
            blocks[a].append((b, B))
        blocks[b].append((a, B.T.copy()))
    for i in range(n):
        M = rng.normal(size=(6, 6))
        D = M @ M.T + 6.0 * np.eye(6) + np.abs(dense[6 * i:6 * i + 6]).sum() * np.eye(6)
        dense[6 * i:6 * i + 6, 6 * i:6 * i + 6] += D
        blocks[i].insert(0, (i, D))
    rp, ci, vals = [0], [], []
    for i in range(n):
        for j, B in blocks[i]:
            ci.append(j)
            vals.append(B)
        rp.append(len(ci))
    b = rng.normal(size=6 * n)
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(vals), b, dense


def test_oracle_linear_solve_matches_dense():
    rp, ci, vals, b, dense = random_block_system()
    x = refcpu.linear_solve(rp, ci, vals, b)
    assert x is not None
    assert np.allclose(x, np.linalg.solve(dense, b), rtol=1e-12, atol=1e-12)


def test_oracle_linear_solve_zero_pivot():
    rp, ci, vals, b, _ = random_block_system(n=3, dup=False)
    vals[0] = 0.0                        # body 0's diagonal block
    assert refcpu.linear_solve(rp, ci, vals, b) is None


def bodies(n):
    sb = scenes.SceneBuilder("blocks")
    for i in range(n):
        sb.add_body(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (float(i), 0.0, 0.0), mass=1.0, inertia=np.eye(3))
    return sb.build(abi.default_settings(), 0.01, 1)


@pytest.mark.gpu
def test_device_linear_solve_matches_oracle():
    from nexdynipc_b200 import runtime
    for seed in range(3):
        rp, ci, vals, b, dense = random_block_system(seed=seed)
        ctx = runtime.Context(bodies(len(rp) - 1))
        xg, st = ctx.linear_solve(rp, ci, vals, b)
        xo = refcpu.linear_solve(rp, ci, vals, b)
        assert np.array_equal(xg, xo), np.abs(xg - xo).max()
        assert st["components"] == 1 and st["singletons"] == 0 and st["largest_component"] == len(rp) - 1
    # a zero pivot is reported, not raised as a fault
    rp, ci, vals, b, _ = random_block_system(n=3, dup=False)
    vals[0] = 0.0
    ctx = runtime.Context(bodies(3))
    with pytest.raises(runtime.NxdError) as e:
        ctx.linear_solve(rp, ci, vals, b)
    assert e.value.status == 3   # NXD_FACTOR_FAILED


@pytest.mark.gpu
def test_eval_all_and_solve_of_the_step_hessian():
    # nxd_eval_all equals the three form calls, and solving the exported
    # total Hessian equals the oracle's solve of the same blocks
    from nexdynipc_b200 import runtime
    sc = scenes.hopper_chains(n_hulls=64, n_chains=4)
    ctx = runtime.Context(sc)
    for _ in range(3):
        ctx.step()
    ow = refcpu.OracleWorld(sc)
    c, _ = ow.detect_contacts()
    x = np.zeros(6 * sc.n_bodies)
    st = ctx.state()
    x[0::6], x[1::6], x[2::6] = st["position"][:, 0], st["position"][:, 1], st["position"][:, 2]
    xh = x.copy()
    ctx.set_form_state(c, None, xh, sc.dt)
    e, g, (rp, ci, vals) = ctx.eval_all(x)
    assert e == ctx.form_value(abi.NXD_FORM_TOTAL, x)
    assert np.array_equal(g, ctx.form_gradient(abi.NXD_FORM_TOTAL, x))
    rp2, ci2, vals2 = ctx.form_hessian_bsr(x)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(vals, vals2)
    xg, stats = ctx.linear_solve(rp, ci, vals.reshape(-1, 36), -g)
    xo = refcpu.linear_solve(rp, ci, vals.reshape(-1, 36), -g)
    assert np.abs(xg - xo).max() <= 1e-12 * max(1.0, np.abs(xo).max())
    assert stats["components"] >= 4
