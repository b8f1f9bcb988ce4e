"""Multi-GPU is replicas only: each rank steps its own scene, and bench.py
combines the ranks' device-timed milliseconds by a max all-reduce. These CPU
tests run that host logic on two gloo ranks (no GPU)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, local = bench._dist()
        assert (w, r, local) == (world, rank, rank)
        ms = 10.0 + 5.0 * rank  # ranks finish at different times
        slowest = bench.max_over_ranks(ms, world, device="cpu")
        out[rank] = (slowest, bench.whole_job_rate(world, 20, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]  # every rank sees the same maximum
    slowest, rate = res[0]
    assert slowest == pytest.approx(15.0)
    assert rate == pytest.approx(2 * 20 / 0.015)  # world * steps / max time


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(12.5, 1) == 12.5
    assert bench.whole_job_rate(1, 10, 100.0) == pytest.approx(100.0)
