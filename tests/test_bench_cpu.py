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


def test_clock_summary_keeps_the_samples_inside_the_timed_region():
    """The nvidia-smi record is filtered by its timestamps: the median clock and the throttle
    reasons come from the samples between the two marks; a region shorter than the sampling
    interval falls back to all samples and says so."""
    import time
    sys.path.insert(0, ROOT)
    import bench
    c = bench.Clocks(0)  # not entered: no nvidia-smi process, the record is written here
    now = time.time()
    for k in range(12):
        t = now - 0.6 + 0.1 * k
        ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        sm = 1965 if k < 4 else 1800                       # idle before, loaded inside
        cap = "Active" if k == 11 else "Not Active"          # power cap only after the region
        c.f.write(f"{ts}, 0, {sm}, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, {cap}\n")
    c.t0, c.t1 = now - 0.25, now + 0.35
    s = c.summary()
    assert s["window"] == "timed region"
    assert s["samples"] == 6 and s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == []
    c.t0, c.t1 = now + 5.0, now + 5.01
    s = c.summary()
    assert s["samples"] == 12 and s["window"].startswith("around")
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_prefers_nvml_samples_inside_the_region():
    """With a (fake) NVML, the polling thread's samples inside the timed region give the clock
    and the reasons, at a rate that fits a region of a few milliseconds."""
    import time
    sys.path.insert(0, ROOT)
    import bench

    class FakeNVML:
        NVML_CLOCK_SM = 1

        def nvmlInit(self):
            pass

        def nvmlDeviceGetHandleByPciBusId(self, bus):
            return bus

        def nvmlDeviceGetMaxClockInfo(self, h, kind):
            return 1965

        def nvmlDeviceGetClockInfo(self, h, kind):
            return 1950

        def nvmlDeviceGetCurrentClocksEventReasons(self, h):
            return 0x4  # sw_power_cap

    c = bench.Clocks("00000000:1b:00.0", nvml=FakeNVML())
    with c:
        c.mark()
        time.sleep(0.05)
        c.mark()
    s = c.summary()
    assert s["window"].startswith("timed region (NVML")
    assert s["samples"] >= 5 and s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
