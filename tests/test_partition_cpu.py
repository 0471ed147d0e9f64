"""One network over two processes, on the CPU: the engine's partition protocol restated in
the oracle and run as two gloo ranks.

Each rank builds the whole network description, simulates its share of every group
(partition.local_range) and, after the update phase of every step, all-gathers the step's
spikes of its neurons over torch.distributed (gloo) and files the other rank's spikes as if
they were emitted locally.  The two shares together must give exactly the spike counts and
membrane potentials of the network simulated by one process.  (The CUDA engine runs the same
protocol once per time batch; tests/test_gpu_partition.py checks it against the whole network
on one GPU.)
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(o):
    sys.path.insert(0, os.path.join(ROOT, "nest-gpu_b200"))
    from workloads import benchmark_network
    neuron, pg = benchmark_network(o, 0.002, 777)   # 2000 neurons, 2e6 synapses
    return neuron


def _rank(rank, world, port, q):
    for sub in ("oracle", "nest-gpu_b200", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle as orc
        from partition import local_range
        o = orc.Oracle()
        neuron = _build(o)

        def exchange(net):
            nodes, heights = net.StepSpikes()
            got = [None] * world
            dist.all_gather_object(got, (nodes.tolist(), heights.tolist()))
            for r, (nn, hh) in enumerate(got):
                if r != rank and nn:
                    net.InjectSpikes(nn, hh)

        o.SetPartition(rank, world, exchange)
        o.Simulate(60.0)
        lo, hi = local_range(len(neuron), rank, world)
        c = np.asarray(o.GetStatus(neuron, "spike_count")).ravel()[lo:hi]
        v = np.float32(np.asarray(o.GetStatus(neuron, "V_m")).ravel())[lo:hi]
        q.put((rank, c.tolist(), v.tolist()))
    finally:
        dist.destroy_process_group()


def test_partitioned_network_equals_whole_on_two_gloo_ranks():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    whole = orc.Oracle()
    neuron = _build(whole)
    whole.Simulate(60.0)
    c_all = np.asarray(whole.GetStatus(neuron, "spike_count")).ravel()
    v_all = np.float32(np.asarray(whole.GetStatus(neuron, "V_m")).ravel())
    assert c_all.sum() > 100
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (c, v)) for r, c, v in (q.get(timeout=600) for _ in ps))
    for p in ps:
        p.join(timeout=120)
    c = np.concatenate([res[0][0], res[1][0]])
    v = np.concatenate([res[0][1], res[1][1]]).astype(np.float32)
    assert np.array_equal(c, c_all)
    assert np.array_equal(v, v_all)
