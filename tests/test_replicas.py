"""The multi-GPU path of bench.py on CPU: one process per rank over a gloo group (world size
2), as `bench.py --gpus 2` runs under torchrun. The model does not shard, so ranks are
independent replicas; the only collective is the MAX all-reduce of their timings, and the
whole-job throughput counts every replica's steps. The reference arm runs on rank 0 alone."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(times[rank], dist)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timings_reduce_to_the_slowest_rank():
    world = 2
    times = [12.5, 17.25]
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), times, out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: 17.25, 1: 17.25}


def test_job_throughput_counts_every_replica():
    import bench
    one = bench.job_throughput(1, 100, 0.26)
    assert bench.job_throughput(2, 100, 0.26) == pytest.approx(2 * one)
    assert one == pytest.approx(100 * bench.DT / 86400.0 / 0.26)
    assert bench.max_over_ranks(3.5) == 3.5     # no group: the rank's own time


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    class Args:
        steps, warmup = 2, 3

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference_arm(Args(), rank=1, world=2)
    assert buf.getvalue() == ""
