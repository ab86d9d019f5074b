"""The multi-process plumbing of bench.py on the CPU: two ranks over gloo
(127.0.0.1), as the benchmark runs them under torchrun.  The path runs replicas
(one job per GPU, no collective on the data path), so what the ranks share is
the timing: every rank reports the slowest rank's time, and only rank 0 runs
and prints the reference arm."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "donof.jl_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(0.25 + rank, dist)            # rank r took 0.25 + r seconds
        dist.barrier()
        # the reference arm's ranks other than 0 return at once, before any work
        line = bench.reference_arm(None, rank, world) if rank != 0 else "rank0"
        out.put((rank, t, line))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_rank_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [1.25, 1.25]        # both ranks see the max
    assert res[1][2] is None                           # rank 1 runs no reference work and prints nothing


def test_single_process_time_is_its_own():
    sys.path[:0] = [str(ROOT)]
    import bench

    assert bench.max_over_ranks(0.5, None) == 0.5
