"""The multi-GPU bench runs independent replicas whose only cross-rank traffic is a barrier
and max / sum reductions of the timed scalars.  Checked here with two gloo ranks on CPU."""
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
