"""The several-GPU path of bench.py is replicas only: every rank steps its
own copy of the scene and the ranks meet only to take the slowest rank's
time.  This checks that host logic with two gloo ranks on the CPU: the
max-over-ranks reduction, the whole-job rate, and the reference arm, which
only rank 0 runs."""
import io
import os
import socket
import sys
import contextlib

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ws, r, local = bench.dist_env()
    # rank r took 10 + r ms: the job's time is the slowest rank's
    t = bench.max_over_ranks(10.0 + rank, device="cpu")
    value = ws * 5 / (t / 1e3)
    # the reference arm: the other ranks return at once and print nothing
    buf = io.StringIO()
    if rank != 0:
        with contextlib.redirect_stdout(buf):
            bench.run_reference(None, ws, r)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(f"{ws} {r} {local} {t} {value} {len(buf.getvalue())}\n")


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    rows = [open(tmp_path / f"r{k}.txt").read().split() for k in range(2)]
    for k, (ws, r, local, t, value, printed) in enumerate(rows):
        assert (int(ws), int(r), int(local)) == (2, k, k)
        assert float(t) == 11.0                     # max over ranks on every rank
        assert float(value) == pytest.approx(2 * 5 / 0.011)
        assert int(printed) == 0


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5
