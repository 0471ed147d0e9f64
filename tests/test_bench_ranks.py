"""Multi-process paths, checked with two gloo ranks on the CPU:
- the replicas of the multi-GPU bench, whose only cross-rank traffic is a barrier and
  max / sum reductions of the timed scalars;
- the spike exchange of a network partitioned over processes (partition.TorchExchange): every
  rank receives every rank's records of a time batch, in rank order;
- the partition of a node group into the ranks' contiguous shares."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        barrier, mx, sm = bench.rank_reducers(dist, "cpu")
        barrier()
        out[rank] = (mx(1.5 + rank), sm(10.0 * (rank + 1)))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
    world, port = 2, 29651
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (2.5, 30.0)


def test_single_process_reducers_are_identities():
    sys.path.insert(0, ROOT)
    import bench
    barrier, mx, sm = bench.rank_reducers(None, "cpu")
    barrier()
    assert mx(3.0) == 3.0 and sm(4.0) == 4.0


def _exchange_worker(rank, world, port, q):
    import os
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from partition import TorchExchange
        ex = TorchExchange(cap=8, device="cpu")
        # this rank's batch: rank + 1 spikes of nodes 100*rank + j at time index 7
        ex.send.zero_()
        s = ex.send.view(-1, 4)
        s[0, 0] = rank + 1
        for j in range(rank + 1):
            s[1 + j] = torch.tensor([100 * rank + j, 0, 7, 0], dtype=torch.int32)
        assert ex._exchange(None) == 0
        r = ex.recv.view(world, 9, 4)
        got = [[int(r[p, 1 + j, 0]) for j in range(int(r[p, 0, 0]))] for p in range(world)]
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_partition_exchange_all_gather_two_ranks():
    """The exchange of a partitioned network over torch.distributed (gloo, two ranks on the
    CPU): every rank receives every rank's spike records in rank order."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_exchange_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    expect = [[0], [100, 101]]
    assert res[0] == expect and res[1] == expect


def test_partition_ranges_cover_groups():
    from partition import local_range
    for n in (1, 7, 1000, 77169):
        for world in (1, 2, 3, 8):
            r = [local_range(n, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
