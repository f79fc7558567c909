"""bench.py's multi-GPU mode, on the CPU: N independent replicas (the path
does not shard; no data-path collective), timed as the slowest rank.  Two
gloo ranks on 127.0.0.1 stand in for two GPUs: each reports its own time,
both must see the maximum, and the whole-job value counts every replica's
atoms over that time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
        out.put((rank, ms, bench.replica_value(1000, 20, world, ms)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_are_timed_as_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [15.0, 15.0]
    # 2 replicas x 1000 atoms x 20 steps in 15 ms
    assert got[0][2] == pytest.approx(2 * 1000 * 20 / 0.015)
