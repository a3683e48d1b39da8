"""The multi-rank bench arithmetic on CPU: two gloo ranks, each with its own
device time, agree on the slowest rank's time and on the whole-job frame rate
(steps x world frames over that time), as bench.py reports under torchrun."""
import os
import socket

import pytest
import torch.multiprocessing as tmp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        agg = bench.whole_job({"b": times[rank][0], "e": times[rank][1]}, 10, world)
        out.put((rank, agg))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_whole_job_is_max_over_ranks(world):
    times = [(0.020, 0.031), (0.025, 0.029)]
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        tb, vb = res[r]["b"]
        te, ve = res[r]["e"]
        assert tb == pytest.approx(0.025) and te == pytest.approx(0.031)
        assert vb == pytest.approx(10 * world / 0.025)
        assert ve == pytest.approx(10 * world / 0.031)


def test_single_rank_needs_no_process_group():
    import bench
    agg = bench.whole_job({"b": 0.5}, 5, 1)
    assert agg["b"] == (0.5, 10.0)
