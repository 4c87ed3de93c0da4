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
    """MeshShape::computeAABB per body; a body without a mesh gets an empty
    box (min > max), which keeps it out of every pair as nxd_body_pairs does."""
    out = np.zeros((sc.n_bodies, 6))
    for i in range(sc.n_bodies):
        v = sc.vertices[sc.vertex_offset[i]:sc.vertex_offset[i + 1]]
        if len(v) == 0 or sc.face_offset[i + 1] == sc.face_offset[i]:
            out[i] = (1.0, 1.0, 1.0, -1.0, -1.0, -1.0)
            continue
        out[i, :3] = v.min(0)
        out[i, 3:] = v.max(0)
    return out


def mixed_meshless():
    """Cubes interleaved with bodies that have no mesh at overlapping poses
    (the reference's meshless pendulum links are such bodies)."""
    from nexdynipc_b200 import abi
    sb = scenes.SceneBuilder("mixed_meshless")
    cv, cf = scenes.box_mesh(0.1, 0.1, 0.1)
    empty_v, empty_f = np.zeros((0, 3)), np.zeros((0, 3), np.int32)
    for k in range(12):
        x = 0.15 * (k % 4)
        y = 0.15 * (k // 4)
        if k % 3 == 1:
            sb.add_body(empty_v, empty_f, (x, y, 0.0), mass=1.0, inertia=np.eye(3))
        else:
            sb.add_body(cv, cf, (x, y, 0.0), quat=scenes.quat_from_axis_angle((0, 1, 1), 0.1 * k))
    return sb.build(abi.default_settings(), 0.01, 1)


@pytest.mark.parametrize("make", [scenes.cube_stack, lambda: scenes.hopper_chains(n_hulls=256, n_chains=4),
                                  mixed_meshless])
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


def test_noalloc_capacity_status_and_bounded_writes():
    # cap one below the pair count: NXD_CAPACITY, the true count, the first
    # cap pairs in order, and nothing written past pairs[2 * cap)
    import ctypes as C
    import torch
    from nexdynipc_b200 import runtime
    sc = scenes.hopper_chains(n_hulls=128, n_chains=2)
    ctx = runtime.Context(sc)
    r = 0.05
    expect = ctx.body_pairs(r)
    assert len(expect) > 2
    dev = torch.device("cuda", torch.cuda.current_device())
    pos = torch.from_numpy(np.ascontiguousarray(sc.position)).to(dev)
    quat = torch.from_numpy(np.ascontiguousarray(sc.orientation)).to(dev)
    lbox = torch.from_numpy(local_boxes(sc)).to(dev)
    cap = len(expect) - 1
    out = torch.full((cap + 64, 2), -7, dtype=torch.int32, device=dev)
    cnt = C.c_int64(0)
    st = runtime.lib().nxd_body_pairs_noalloc(C.c_void_p(pos.data_ptr()), C.c_void_p(quat.data_ptr()),
                                              C.c_void_p(lbox.data_ptr()), sc.n_bodies, r,
                                              C.c_void_p(out.data_ptr()), cap, C.byref(cnt), None)
    assert st == 4                                  # NXD_CAPACITY
    assert cnt.value == len(expect)
    got = out.cpu().numpy()
    assert np.array_equal(got[:cap], expect[:cap])
    assert (got[cap:] == -7).all()
