"""bench.py's multi-rank plumbing on CPU: two gloo ranks, each an independent replica
with its own timings, agree on the element-wise maximum, and the whole-job rate counts
every rank's units over the slowest rank's time."""

import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: step 4 + r ms, kernel 3.5 - r ms, e2e 5 + 2r ms
        got = bench.max_over_ranks(dist, [4.0 + rank, 3.5 - rank, 5.0 + 2 * rank], "cpu")
        out[rank] = got + [bench.whole_job_rate(world, 1000, got[0])]
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    step, kern, e2e, rate = res[0]
    assert (step, kern, e2e) == (5.0, 3.5, 7.0)
    assert rate == pytest.approx(2 * 1000 / 5e-3)


def test_single_process_keeps_its_values():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, [1, 2.5], "cpu") == [1.0, 2.5]
    assert bench.whole_job_rate(1, 10, 2.0) == pytest.approx(5000.0)
