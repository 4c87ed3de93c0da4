"""The zero-allocation broad-phase entry point against nxd_body_pairs.

nxd_body_pairs_noalloc serves callers that cannot allocate device memory
(their engine hands out every device byte from its own pool, or runs under a
cap that forbids allocator calls after start-up): they pass device buffers
they own, and the library's fixed scratch array does the rest.  The pairs it
returns must equal those of the ordinary entry point, index for index and in
the same order, on two calls in a row (the second call sees the scratch the
first one left behind).
"""
import numpy as np
import pytest

from nexdynipc_b200 import scenes

pytestmark = pytest.mark.gpu


def local_boxes(sc):
    out = np.zeros((sc.n_bodies, 6))
    for i in range(sc.n_bodies):
        v = sc.vertices[sc.vertex_offset[i]:sc.vertex_offset[i + 1]]
        out[i, :3] = v.min(0)
        out[i, 3:] = v.max(0)
    return out


@pytest.mark.parametrize("make", [scenes.cube_stack, lambda: scenes.hopper_chains(n_hulls=256, n_chains=4)])
def test_noalloc_pairs_match_body_pairs(make):
    import torch
    from nexdynipc_b200 import runtime
    sc = make()
    ctx = runtime.Context(sc)
    dev = torch.device("cuda", torch.cuda.current_device())
    pos = torch.from_numpy(np.ascontiguousarray(sc.position)).to(dev)
    quat = torch.from_numpy(np.ascontiguousarray(sc.orientation)).to(dev)
    lbox = torch.from_numpy(local_boxes(sc)).to(dev)
    cap = 4 * sc.n_bodies * 16
    out = torch.full((cap, 2), -1, dtype=torch.int32, device=dev)
    for r in (sc.settings.dhat, 0.05):
        expect = ctx.body_pairs(r)
        for call in range(2):
            out.fill_(-1)
            n = runtime.body_pairs_noalloc(pos.data_ptr(), quat.data_ptr(), lbox.data_ptr(), sc.n_bodies, r,
                                           out.data_ptr(), cap)
            got = out[:n].cpu().numpy()
            assert n == len(expect), (r, call)
            assert np.array_equal(got, expect), (r, call)


def test_noalloc_rejects_oversize():
    from nexdynipc_b200 import runtime
    with pytest.raises(runtime.NxdError):
        runtime.body_pairs_noalloc(1, 1, 1, 16385, 0.0, 1, 1)
