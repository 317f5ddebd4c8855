"""Multi-rank host logic of bench.py on CPU with gloo (world size 2): every rank runs its
own case (weak scaling, no collective on the data path) and the timing is the max over
ranks.  No GPU is used."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        p = bench.rank_workload(bench.workload(1 << 10), rank)
        out[rank] = (bench.reduce_max(10.0 + 5.0 * rank), p.seed)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_distinct_cases():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(120)
        assert pr.exitcode == 0
    assert out[0][0] == out[1][0] == 15.0          # max over ranks on every rank
    assert out[0][1] != out[1][1]                   # each rank traces its own case


def test_single_process_reduce_is_identity():
    import bench
    assert bench.reduce_max(3.5) == 3.5
