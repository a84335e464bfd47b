"""The multi-process path of bench.py on CPU: two gloo ranks, each timing its own replica; the
whole-job value is all ranks' steps over the slowest rank's time, and every rank agrees on it."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms_local = 100.0 * (rank + 1)        # rank 1 is the slower replica
    value, ms = bench.replica_value(dist, world, 8, ms_local)
    launches = bench.sum_over_ranks(dist, 10.0 * (rank + 1))
    bench.barrier(dist)
    out[rank] = (value, ms, launches)
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_bench():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        value, ms, launches = res[r]
        assert ms == 200.0                         # max over ranks
        assert value == pytest.approx(2 * 8 / 0.2)  # all ranks' steps / slowest time
        assert launches == 30.0
