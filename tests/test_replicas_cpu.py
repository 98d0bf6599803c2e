"""The bench's N>1 path on CPU: two gloo ranks (127.0.0.1) agree on the slowest
rank's time and on the whole-job rate, as bench.py computes them under torchrun."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = [10.0, 25.0][rank]
    m = bench.max_over_ranks(ms, dist, device="cpu")
    rate = bench.job_rate(world, 64 ** 3, 5, m)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, rate))


def test_two_rank_aggregation_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [25.0, 25.0]
    expect = 2 * 64 ** 3 * 3 * 5 / 0.025
    assert all(r[2] == pytest.approx(expect) for r in res)


def test_single_rank_aggregation_is_identity():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(1, 8, 2, 1000.0) == 8 * 3 * 2
