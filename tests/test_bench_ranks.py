"""Multi-rank path of bench.py on CPU: two gloo ranks (127.0.0.1) exercise the
max-over-ranks timing reduction, the whole-job value of independent replicas,
and the reference arm's rank gating (only rank 0 runs and prints)."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # rank r took 10 + r ms per step on its replica
        ms = bench.max_over_ranks(10.0 + rank, world)
        value = bench.job_value(1000, world, ms)
        # the reference arm runs on rank 0 only; other ranks return at once
        ran = None
        if rank != 0:
            args = type('A', (), dict(small=True, steps=1, warmup=0, gpus=world))()
            ran = bench.run_reference(args, rank, world)
        out.put((rank, ms, value, ran))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_driver():
    world = 2
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, ran in res:
        assert ms == pytest.approx(11.0)                 # the slowest rank bounds the job
        assert value == pytest.approx(1000 * 2 / 11e-3)  # all ranks' cells / that time
    assert res[1][3] is None                             # rank 1 did no reference work


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_value(100, 1, 2.0) == pytest.approx(5e4)
