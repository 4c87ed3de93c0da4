"""Failure detection of the Newton solve's grid barrier, without a GPU fault.

The solve's CTAs meet at grid barriers whose waits are bounded; a wait that
runs out sets NXD_TIMEOUT and every CTA returns.  nxd_debug_grid_wait makes
that happen on purpose: a small poll limit, and the last CTA kept away from
its first barrier (by a bounded wait of its own) until the others give up.
The step must then report NXD_TIMEOUT, and the context must stay usable:
after the hook is cleared and the state set again, it steps exactly as a
fresh context.  With the bounded global barrier and no CTA held, the step
must equal the cluster-barrier step bit for bit.  The reference has no such
report: a failed solve leaves Newton's iterate in place silently
(src/Math/NewtonSolver.cpp:43-46).
"""
import numpy as np
import pytest

from nexdynipc_b200 import scenes

pytestmark = pytest.mark.gpu

NXD_TIMEOUT = 6


def scene():
    # 147 bodies: 882 DOFs, a two-CTA Newton grid
    return scenes.hopper_chains(n_hulls=128, n_chains=2)


def test_held_cta_times_out_and_context_recovers():
    from nexdynipc_b200 import runtime
    sc = scene()
    ctx = runtime.Context(sc)
    init = sc.initial_state()
    ctx.debug_grid_wait(2000, True)
    ctx.step()
    assert ctx.diagnostics()["status"] == NXD_TIMEOUT
    ctx.debug_grid_wait(0, False)
    assert ctx.diagnostics()["status"] == 0
    ctx.set_state(init)
    fresh = runtime.Context(sc)
    for _ in range(3):
        ctx.step()
        fresh.step()
        assert ctx.diagnostics()["status"] == 0
    a, b = ctx.state(), fresh.state()
    assert np.abs(a["position"] - b["position"]).max() <= 1e-9
    assert np.abs(a["orientation"] - b["orientation"]).max() <= 1e-9


def test_bounded_global_barrier_matches_cluster_barrier():
    from nexdynipc_b200 import runtime
    sc = scene()
    ctx = runtime.Context(sc)
    ctx.debug_grid_wait(1 << 20, False)
    ref = runtime.Context(sc)
    for _ in range(5):
        ctx.step()
        ref.step()
    assert ctx.diagnostics()["status"] == 0
    a, b = ctx.state(), ref.state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_hook_argument_checks():
    from nexdynipc_b200 import runtime
    ctx = runtime.Context(scene())
    with pytest.raises(runtime.NxdError):
        ctx.debug_grid_wait(0, True)          # a hold needs a poll limit
    with pytest.raises(runtime.NxdError):
        ctx.debug_grid_wait((1 << 20) + 1, False)
