"""The multi-GPU form is replicas only: every rank runs its own copy of the
workload and the job's throughput is the ranks' total over the slowest
rank's device time.  The rank logic of bench.py, run as two gloo ranks on
the CPU."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = [3.0, 5.0][rank]
        ms = bench.max_over_ranks(ms_local, dist, device="cpu")
        value = bench.replica_throughput(world, 1024, 10, ms)
        t = torch.tensor([ms, value], dtype=torch.float64)
        g = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(g, t)
        if rank == 0:
            out.put([x.tolist() for x in g])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1]                      # every rank agrees
    ms, value = res[0]
    assert ms == 5.0                             # the slowest replica
    assert value == pytest.approx(2 * 1024 * 10 / 5e-3)


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(4.0) == 4.0
    assert bench.replica_throughput(1, 1024, 100, 100.0) == pytest.approx(1.024e6)
