"""One network over several partitions (one process per GPU in production), on one GPU.

`partition.LoopbackExchange` runs `world` partitions of the same network in threads of this
process, each with its own engine, exchanging the spikes of every time batch through host
barriers and device copies (no kernel waits for another partition).  Every partition
simulates its share of every node group; together they must give exactly the spikes, events
and state of the whole network simulated by one engine.
"""
import numpy as np
import pytest

import nestgpu as ngpu
from partition import LoopbackExchange, local_range
from workloads import balanced_network, benchmark_network, microcircuit

pytestmark = pytest.mark.gpu


def gather(parts, sizes):
    """Concatenate every partition's own share of the per-neuron arrays of each group."""
    world = len(parts)
    out = []
    for gi, n in enumerate(sizes):
        pieces = []
        for r in range(world):
            lo, hi = local_range(n, r, world)
            pieces.append(parts[r][gi][lo:hi])
        out.append(np.concatenate(pieces))
    return out


def run_split(build, world, t_ms, read):
    """Partitioned run; read() returns a list of per-group arrays (full length)."""
    lb = LoopbackExchange(world, cap=1 << 15)
    state = {}

    def b(r):
        state[r] = build()

    def sim(r):
        ngpu.Simulate(t_ms)
        st = ngpu.GetStats()
        return read(state[r]), st["n_events"], st["status"]

    res = lb.run(b, sim)
    return [x[0] for x in res], sum(x[1] for x in res), [x[2] for x in res]


def run_whole(build, t_ms, read):
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    groups = build()
    ngpu.Simulate(t_ms)
    st = ngpu.GetStats()
    out = read(groups)
    ngpu.Reset()
    return out, st["n_events"]


def counts_and_vm(groups):
    out = []
    for g in groups:
        out.append(np.asarray(ngpu.GetStatus(g, "spike_count")).ravel())
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_benchmark_network_equals_whole(world):
    """The benchmark network at 1% size (generated per-target blocks, one Poisson generator):
    spike counts, membrane potentials and events of the partitions equal the whole run."""
    def build():
        neuron, pg = benchmark_network(ngpu, 0.01, 20240)
        return [neuron]

    def read(groups):
        g = groups[0]
        return [np.asarray(ngpu.GetStatus(g, "spike_count")).ravel(),
                np.float32(np.asarray(ngpu.GetStatus(g, "V_m")).ravel())]

    whole, ev_whole = run_whole(build, 200.0, read)
    parts, ev_parts, status = run_split(build, world, 200.0, read)
    n = len(whole[0])
    c = gather([[p[0]] for p in parts], [n])[0]
    v = gather([[p[1]] for p in parts], [n])[0]
    assert whole[0].sum() > 1000
    assert np.array_equal(c, whole[0])
    assert np.array_equal(v, whole[1])
    assert ev_parts == ev_whole
    assert status == [0] * world


def test_partitioned_microcircuit_equals_whole():
    """The microcircuit slice (eight iaf_psc_exp groups in one launch, every projection
    expanded on the device, normal-clipped delays from one step): same spikes."""
    def build():
        ngpu.SetDeviceRuleMinEdges(0)
        return microcircuit(ngpu, scale=0.03)

    whole, ev_whole = run_whole(build, 150.0, counts_and_vm)
    parts, ev_parts, status = run_split(build, 2, 150.0, counts_and_vm)
    sizes = [len(x) for x in whole]
    got = gather(parts, sizes)
    assert sum(x.sum() for x in whole) > 1000
    for a, b in zip(got, whole):
        assert np.array_equal(a, b)
    assert ev_parts == ev_whole and status == [0, 0]


def test_partitioned_balanced_network_with_records_equals_whole():
    """The balanced network as specified (host-store connections drawn by the reference's
    fixed_indegree rule, 400 Poisson generators): spike counts and the recorded V_m of neurons
    owned by either partition."""
    rec_nodes = [0, 1, 799, 800, 999]

    def build():
        neuron = balanced_network(ngpu, seed=42, drive="poisson")
        ngpu.CreateRecord("", ["V_m"] * len(rec_nodes), [neuron[i] for i in rec_nodes], [0] * len(rec_nodes))
        return [neuron]

    def read(groups):
        return [np.asarray(ngpu.GetStatus(groups[0], "spike_count")).ravel(),
                np.float32(np.asarray(ngpu.GetRecordData(0), dtype=np.float64))]

    whole, _ = run_whole(build, 300.0, read)
    parts, _, status = run_split(build, 2, 300.0, read)
    n = len(whole[0])
    assert np.array_equal(gather([[p[0]] for p in parts], [n])[0], whole[0])
    for col, node in enumerate(rec_nodes):
        owner = 0 if node < local_range(n, 0, 2)[1] else 1
        assert np.array_equal(parts[owner][1][:, 1 + col], whole[1][:, 1 + col])
    assert status == [0, 0]
