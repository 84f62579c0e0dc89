"""bench.py's multi-rank plumbing on the CPU: two gloo ranks (127.0.0.1) take the maximum of
their per-rank times through the same helper that the GPU runs use under torchrun, after a
barrier, as every rank must."""
import datetime
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    v = bench.reduce_max_over_ranks(1.5 + rank, world, "cpu")
    same = bench.reduce_max_over_ranks(7.0, world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, v, same))


def test_reduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _, _ in got) == [0, 1]
    assert all(v == 2.5 and same == 7.0 for _, v, same in got), got


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max_over_ranks(3.25, 1, "cpu") == 3.25
