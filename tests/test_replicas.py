"""The N > 1 path of bench.py on CPU: independent replicas whose job time is
the slowest rank's, reduced with torch.distributed (gloo, world size 2)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (r + 1) * 10 ms for the device part and 100 - r ms end to end
        ms, ems = bench.max_over_ranks([10.0 * (rank + 1), 100.0 - rank], torch.device("cpu"), world)
        q.put((rank, ms, ems, bench.replica_rate(1e12, ms, world)))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, ems, rate in got:
        assert ms == 20.0 and ems == 100.0                 # every rank sees the slowest rank's times
        assert rate == pytest.approx(2 * 1e12 / 20e-3)     # whole-job work over the job's time


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks([3.0, 4.0], None, 1) == [3.0, 4.0]
    assert bench.replica_rate(5.0, 1000.0, 1) == pytest.approx(5.0)
