"""Block-Jacobi PCG on a 6x6-block BSR matrix (nxd_pcg_solve) against the
direct block LDL^T of the oracle, plus a large banded system checked by its
residual."""
import numpy as np
import pytest

from nexdynipc_b200 import abi, scenes
from oracle import refcpu

pytestmark = pytest.mark.gpu


def small_context():
    sb = scenes.SceneBuilder("one")
    sb.add_body(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (0.0, 0.0, 0.0), mass=1.0, inertia=np.eye(3))
    from nexdynipc_b200 import runtime
    return runtime.Context(sb.build(abi.default_settings(), 0.01, 1))


def banded_system(n, offsets=(1, 64, 4096), seed=0, scale=0.1):
    """SPD block matrix: body i coupled to i +- o for o in offsets, random
    off-diagonal blocks (B and B^T), diagonally dominant diagonal blocks."""
    rng = np.random.default_rng(seed)
    rows, cols, blks = [np.arange(n)], [np.arange(n)], []
    M = rng.normal(size=(n, 6, 6)) * 0.05
    D = np.einsum("nij,nkj->nik", M, M) + (1.0 + 2 * len(offsets) * 6 * scale) * np.eye(6)
    blks.append(D)
    for o in offsets:
        if o >= n:
            continue
        i = np.arange(n - o)
        B = rng.uniform(-scale, scale, size=(n - o, 6, 6))
        rows += [i, i + o]
        cols += [i + o, i]
        blks += [B, np.transpose(B, (0, 2, 1))]
    r, c, v = np.concatenate(rows), np.concatenate(cols), np.concatenate(blks)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp).astype(np.int32), c.astype(np.int32), np.ascontiguousarray(v.reshape(-1, 36))


def bsr_matvec(rp, ci, vals, x):
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    y = np.einsum("kij,kj->ki", vals.reshape(-1, 6, 6), x.reshape(-1, 6)[ci])
    out = np.zeros((n, 6))
    np.add.at(out, rows, y)
    return out.reshape(-1)


def test_pcg_matches_direct_solve():
    ctx = small_context()
    rp, ci, vals = banded_system(300, offsets=(1, 7, 40), seed=3)
    b = np.random.default_rng(1).normal(size=6 * 300)
    x, st = ctx.pcg_solve(rp, ci, vals, b, tol=1e-13, max_iter=500)
    xo = refcpu.linear_solve(rp, ci, vals, b)
    assert st["rc"] == 0 and st["status"] == 0 and st["relative_residual"] <= 1e-13
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()
    # a second call on the same context gives the same bits (fixed-tree sums)
    x2, _ = ctx.pcg_solve(rp, ci, vals, b, tol=1e-13, max_iter=500)
    assert np.array_equal(x, x2)


def test_pcg_iteration_cap_and_bad_matrix():
    ctx = small_context()
    rp, ci, vals = banded_system(100, offsets=(1, 9), seed=4)
    b = np.ones(600)
    x, st = ctx.pcg_solve(rp, ci, vals, b, tol=1e-15, max_iter=2, check=False)
    assert st["rc"] == 1 and st["iterations"] == 2            # NXD_NOT_CONVERGED
    bad = vals.copy()
    bad[0] = 0.0                                             # a zero diagonal block
    from nexdynipc_b200 import runtime
    with pytest.raises(runtime.NxdError) as e:
        ctx.pcg_solve(rp, ci, bad, b)
    assert e.value.status == 3                               # NXD_FACTOR_FAILED


def test_pcg_large_banded_system():
    ctx = small_context()
    n = 60000
    rp, ci, vals = banded_system(n, seed=5)
    b = np.random.default_rng(2).normal(size=6 * n)
    x, st = ctx.pcg_solve(rp, ci, vals, b, tol=1e-12, max_iter=400)
    assert st["rc"] == 0
    r = bsr_matvec(rp, ci, vals, x) - b
    assert np.linalg.norm(r) <= 1e-11 * np.linalg.norm(b)
    assert st["grid"] > 1


def test_pcg_reads_the_upper_block_triangle():
    # the lower triangle is not read: zeroing it changes no bit of the
    # solution; duplicate upper blocks are summed; a block without its
    # transposed partner is rejected
    ctx = small_context()
    rp, ci, vals = banded_system(200, offsets=(1, 5, 33), seed=6)
    b = np.random.default_rng(3).normal(size=6 * 200)
    x, st = ctx.pcg_solve(rp, ci, vals, b, tol=1e-13, max_iter=500)
    rows = np.repeat(np.arange(200), np.diff(rp))
    low = vals.copy()
    low[ci < rows] = 0.0
    low[ci == rows] = np.triu(vals[ci == rows].reshape(-1, 6, 6)).reshape(-1, 36)
    x2, _ = ctx.pcg_solve(rp, ci, low, b, tol=1e-13, max_iter=500)
    assert np.array_equal(x, x2)
    # split every upper block into two halves stored side by side
    up = ci > rows
    k_up = np.nonzero(up)[0]
    rp3 = rp.copy()
    for r in rows[k_up]:
        rp3[r + 1:] += 1
    order = np.argsort(np.concatenate([np.arange(len(ci)), k_up]), kind="stable")
    ci3 = np.concatenate([ci, ci[k_up]])[order].astype(np.int32)
    v3 = np.concatenate([np.where(up[:, None], 0.5 * vals, vals), 0.5 * vals[k_up]])[order]
    x3, _ = ctx.pcg_solve(rp3, ci3, np.ascontiguousarray(v3), b, tol=1e-13, max_iter=500)
    assert np.abs(x3 - x).max() <= 1e-12 * np.abs(x).max()
    # drop one block below the diagonal: the pattern is no longer symmetric
    from nexdynipc_b200 import runtime
    k = int(np.nonzero(ci < rows)[0][5])
    keep = np.ones(len(ci), bool)
    keep[k] = False
    rp4 = rp.copy()
    rp4[rows[k] + 1:] -= 1
    with pytest.raises(runtime.NxdError) as e:
        ctx.pcg_solve(rp4, ci[keep], np.ascontiguousarray(vals[keep]), b)
    assert e.value.status == 7                               # NXD_INVALID_ARGUMENT
