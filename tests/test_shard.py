"""Independent scenes sharded over ranks (nexdynipc_b200/shard.py): the
greedy assignment covers every scene once and keeps the ranks balanced, and
two gloo ranks on the CPU, each stepping its share (here with the CPU
oracle, the device's checker), gather exactly the results one process gets
stepping all scenes."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_assignment_covers_and_balances():
    from nexdynipc_b200 import scenes, shard
    scs = scenes.batched_scenes()
    costs = [shard.scene_cost(s) for s in scs]
    for ws in (1, 2, 3, 4, 8):
        parts = shard.assign(costs, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(scs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # greedy LPT: no rank more than one scene's cost above the mean
        assert max(loads) - np.mean(loads) <= max(costs) + 1e-9
        assert parts == shard.assign(costs, ws)          # deterministic
    with pytest.raises(ValueError):
        shard.assign(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_results(scs, idx, steps):
    from oracle import refcpu
    out = {}
    for i in idx:
        ow = refcpu.OracleWorld(scs[i])
        for _ in range(steps):
            ow.step()
        out[i] = {"position": ow.state()["position"], "n_contacts": ow.diagnostics()["n_contacts"]}
    return out


def _rank(rank, world, port, out_dir):
    import datetime
    import pickle
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from nexdynipc_b200 import scenes, shard
    scs = scenes.batched_scenes(n_scenes=10)
    idx, _ = shard.my_scenes(scs, rank, world)
    res = shard.gather(_oracle_results(scs, idx, 3), len(scs))
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.pkl"), "wb") as f:
        pickle.dump((idx, res), f)


def test_two_gloo_ranks_gather(tmp_path):
    import pickle
    import torch.multiprocessing as mp
    from nexdynipc_b200 import scenes
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    got = [pickle.load(open(tmp_path / f"r{k}.pkl", "rb")) for k in range(2)]
    (i0, r0), (i1, r1) = got
    assert sorted(i0 + i1) == list(range(10)) and not set(i0) & set(i1)
    scs = scenes.batched_scenes(n_scenes=10)
    want = _oracle_results(scs, range(10), 3)
    for res in (r0, r1):                 # every rank receives the whole list
        assert len(res) == 10
        for i, r in enumerate(res):
            assert np.array_equal(r["position"], want[i]["position"])
            assert r["n_contacts"] == want[i]["n_contacts"]


def test_gather_single_process_and_errors():
    from nexdynipc_b200 import shard
    assert shard.gather({1: "b", 0: "a"}, 2) == ["a", "b"]
    with pytest.raises(RuntimeError):
        shard.gather({0: "a"}, 2)
