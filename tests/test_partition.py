"""Mesh partitions on the host: the recursive coordinate bisection and the
halo plans (zj_partition, zj_halo_plan), and the exchange protocol the plans
define, run by two gloo ranks on the CPU: each rank sends its side of every
cut face's trace rows, group by group in the plan's order, and receives the
other side's into its ghost rows -- the rows a multi-process run moves with
NCCL send/recv, and the single-process driver (zj_parts_*) with peer
copies."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from zhijian_b200 import meshgen as M
from zhijian_b200 import partition as PT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nparts", [1, 2, 3, 5, 8])
def test_partition_is_balanced_and_deterministic(zjlib, nparts):
    mesh = M.tgv_mesh(24, seed=1)
    p = PT.partition(mesh, nparts)
    assert p.shape == (mesh.n_elem,) and p.min() == 0 and p.max() == nparts - 1
    counts = np.bincount(p, minlength=nparts)
    assert counts.max() - counts.min() <= 1
    assert np.array_equal(p, PT.partition(mesh, nparts))


def test_partition_of_a_curved_and_a_mixed_mesh(zjlib):
    for mesh in (M.curved_quads(6, 5, 2, 0.0, 1.0, 0.0, 1.0, 0.04), M.split_quads(M.tgv_mesh(8, seed=1), 0.3, 3)):
        p = PT.partition(mesh, 4)
        assert np.bincount(p).max() - np.bincount(p).min() <= 1


def test_halo_plans_match_across_every_cut(zjlib):
    mesh = M.tgv_mesh(16, seed=1)
    n = 4
    p = PT.partition(mesh, n)
    plans = [PT.halo_plan(mesh, p, r) for r in range(n)]
    for r, pl in enumerate(plans):
        assert np.array_equal(np.sort(pl["elems"]), np.flatnonzero(p == r))
        assert np.all(np.diff(pl["nbr"]) > 0) and r not in pl["nbr"]
        assert np.all(p[pl["mine"] // 4] == r)
        for i, q in enumerate(pl["nbr"]):
            a, b = pl["off"][i], pl["off"][i + 1]
            assert np.all(np.diff(pl["face"][a:b]) > 0)          # global face order
            assert np.all(p[pl["remote"][a:b] // 4] == q)
            other = plans[q]
            j = int(np.flatnonzero(other["nbr"] == r)[0])
            c, d = other["off"][j], other["off"][j + 1]
            assert np.array_equal(pl["face"][a:b], other["face"][c:d])
            assert np.array_equal(pl["mine"][a:b], other["remote"][c:d])
            assert np.array_equal(pl["remote"][a:b], other["mine"][c:d])
    # every interior face the partition cuts appears once on each side
    total = sum(len(pl["face"]) for pl in plans)
    assert total % 2 == 0 and total > 0


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


N1 = 4   # points per edge (P3)


def global_rows(n_elem):
    """A stand-in for the traces: row element*4 + edge holds N1 points x 4
    variables with values no two rows share."""
    slot = np.arange(n_elem * 4, dtype=np.float64)[:, None, None]
    return slot * 100.0 + np.arange(N1)[None, :, None] * 10.0 + np.arange(4)[None, None, :] * 0.5


def rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from zhijian_b200 import meshgen as M
    from zhijian_b200 import partition as PT
    mesh = M.tgv_mesh(12, seed=1)
    p = PT.partition(mesh, world)
    pl = PT.halo_plan(mesh, p, rank)
    rows = global_rows(mesh.n_elem)            # this rank reads only its own rows
    ghost = np.full((len(pl["face"]), N1, 4), np.nan)
    reqs = []
    for i, q in enumerate(pl["nbr"]):
        a, b = pl["off"][i], pl["off"][i + 1]
        send = torch.from_numpy(np.ascontiguousarray(rows[pl["mine"][a:b]]))
        recv = torch.empty(send.shape, dtype=torch.float64)
        reqs.append((dist.isend(send, int(q)), dist.irecv(recv, int(q)), a, b, recv, send))
    for s, r, a, b, recv, _ in reqs:
        s.wait()
        r.wait()
        ghost[a:b] = recv.numpy()
    ok = bool(np.array_equal(ghost, rows[pl["remote"]]))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ok, len(pl["face"])))


def test_two_gloo_ranks_exchange_their_cut_traces():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert all(ok for _, ok, _ in res)
    assert res[0][2] == res[1][2] > 0
