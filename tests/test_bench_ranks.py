"""The benchmark's multi-rank path on the CPU: two gloo ranks run the same
Ranks helper the bench runs with NCCL (process group from the torchrun
environment, barrier, maximum over ranks), the whole-job rate counts every
rank's units over the slowest rank's time, and the reference arm runs on rank
0 alone while the other ranks return without work."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench
    r = bench.Ranks("gloo", timeout_s=30)
    assert (r.world, r.rank) == (world, rank)
    r.barrier()
    slowest = r.max(10.0 * (rank + 1))            # per-rank milliseconds
    rate = bench.whole_job_rate(1000.0, r.world, slowest)

    class Args:
        steps, warmup, gpus, run_seconds = 1, 0, world, 0.2
    ref = bench.run_reference(Args)
    r.barrier()
    r.close()
    out.put((rank, slowest, rate, None if ref is None else (ref["impl"], ref["n_gpus"])))


def test_two_gloo_ranks():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[1] for x in res] == [20.0, 20.0]                  # the slowest rank, on both
    assert all(x[2] == pytest.approx(2 * 1000.0 / 0.020) for x in res)
    assert res[0][3] == ("reference", 2)                        # rank 0 times the reference arm
    assert res[1][3] is None                                     # rank 1 does no work
