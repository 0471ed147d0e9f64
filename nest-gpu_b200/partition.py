"""One network over several processes, one GPU each.

Every process builds the same network description (the same Create / Connect calls and
seeds, so every rank draws the same connections), then declares its share with
`SetPartition(rank, world)` before calibration: it simulates neurons
floor(n*rank/world) .. floor(n*(rank+1)/world)-1 of every node group, and its delivery
layout holds only the in-edges of those neurons (generated blocks draw only those targets'
edges; rule-based calls expanded on the device skip the other targets).  After each time
batch (at most the minimum delay in steps, so no spike emitted inside a batch can reach a
target inside it) the engine hands the batch's spikes of its own neurons to an exchange
function; the other processes' spikes then enter its spike ring, as the reference's MPI
exchange does once per step (src/spike_mpi.cu:291-370).

Exchange buffers: int32 device tensors of (cap + 1) records of 4 ints per process:
record 0 holds the count, record 1 + j = (source node, height bits, time index, 0).
`TorchExchange` all-gathers them over torch.distributed (NCCL between GPUs);
`LoopbackExchange` runs several partitions in threads of one process (one GPU), for
tests.  Results are read per process for its own neurons (`local_range`).
"""
import threading

import nestgpu as ngpu


def local_range(n, rank, world):
    """Neurons of a group of n simulated by process `rank` of `world` (relative indices)."""
    return (n * rank) // world, (n * (rank + 1)) // world


class TorchExchange(object):
    """All-gather of the exchange buffers over torch.distributed (one process per GPU)."""

    def __init__(self, cap=1 << 16, device="cuda", group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.cap = cap
        self.send = torch.zeros((cap + 1) * 4, dtype=torch.int32, device=device)
        self.recv = torch.zeros(self.world * (cap + 1) * 4, dtype=torch.int32, device=device)
        self._fn = ngpu.EXCHANGE_FN(self._exchange)

    def _exchange(self, user):
        try:
            self.dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
            if self.recv.is_cuda:
                self.torch.cuda.current_stream().synchronize()
            return 0
        except Exception:
            return 1

    def attach(self):
        """Declare this process's share and the exchange (before calibration)."""
        ngpu.SetPartition(self.rank, self.world)
        ngpu.SetExchange(self.send.data_ptr(), self.recv.data_ptr(), self.cap, self._fn)


class LoopbackExchange(object):
    """`world` partitions of one network in threads of one process on one GPU.  Each thread
    owns an engine (the engine is per thread); the exchange is a barrier, copies of every
    partition's send buffer into every receive buffer, and a second barrier.  Nothing on the
    GPU waits for another partition: the waits are host barriers between batches."""

    def __init__(self, world, cap=1 << 16, device="cuda"):
        import torch
        self.torch = torch
        self.world, self.cap = world, cap
        self.send = [torch.zeros((cap + 1) * 4, dtype=torch.int32, device=device) for _ in range(world)]
        self.recv = [torch.zeros(world * (cap + 1) * 4, dtype=torch.int32, device=device) for _ in range(world)]
        self.barrier = threading.Barrier(world, timeout=600)
        self._fns = [ngpu.EXCHANGE_FN(lambda user, r=r: self._exchange(r)) for r in range(world)]

    def _exchange(self, r):
        try:
            self.barrier.wait()
            blk = (self.cap + 1) * 4
            for q in range(self.world):
                self.recv[r][q * blk:(q + 1) * blk].copy_(self.send[q])
            self.torch.cuda.synchronize()
            self.barrier.wait()
            return 0
        except Exception:
            self.barrier.abort()
            return 1

    def attach(self, rank):
        """Declare partition `rank` on the calling thread's engine (before calibration)."""
        ngpu._c["NESTGPU_SetOnException"](1)
        ngpu.SetPartition(rank, self.world)
        ngpu.SetExchange(self.send[rank].data_ptr(), self.recv[rank].data_ptr(), self.cap, self._fns[rank])

    def run(self, build, simulate):
        """Run build(rank) (creates the network on the thread's engine; its calls are
        serialised) and then simulate(rank) for every partition in its own thread; returns
        the list of simulate's results."""
        lock = threading.Lock()
        out = [None] * self.world
        err = []

        def worker(r):
            try:
                with lock:
                    ngpu._c["NESTGPU_SetOnException"](1)
                    ngpu.SetVerbosityLevel(0)
                    build(r)
                    self.attach(r)
                out[r] = simulate(r)
            except BaseException as e:   # reported to the caller
                err.append(e)
                self.barrier.abort()
            finally:
                try:
                    ngpu.Reset()
                except Exception:
                    pass

        th = [threading.Thread(target=worker, args=(r,)) for r in range(self.world)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if err:
            raise err[0]
        return out
