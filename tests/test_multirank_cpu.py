"""The N>1 bench path (one replica per GPU, replicas only): per-rank seeds, the
max-over-ranks job time and the whole-job rate, run as two gloo ranks on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        ms = 10.0 + rank  # rank 1 is slower
        job_ms = bench.max_over_ranks(ms, dist, "cpu")
        out.put((rank, bench.rank_seed(rank), job_ms, bench.job_gbs(64 << 20, world, job_ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_rate():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, seed0, ms0, gbs0), (r1, seed1, ms1, gbs1) = res
    assert seed0 != seed1  # each replica has its own stripes
    assert ms0 == ms1 == 11.0  # the job takes as long as its slowest rank
    assert gbs0 == gbs1 == pytest.approx(2 * (64 << 20) / 11e-3 / 1e9)
