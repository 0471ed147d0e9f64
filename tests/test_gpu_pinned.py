"""Parity of the networks the benchmarks simulate, at sizes the oracle finishes in seconds.

- The 1M-neuron benchmark network (bench.py) at 1% size, built by the same code
  (workloads.benchmark_network: the generated per-target fixed in-degree rule): the
  engine's delivery layout holds exactly the oracle's edges, segment by segment, and
  200 ms give the same spike counts, events and membrane state.
- The plain small balanced network exactly as specified (seed 42, 1000 neurons, the
  reference's fixed_indegree rule, 400 Poisson generators at 10 Hz, 1 s): the same spike
  counts and recorded V_m / w traces as the oracle; its fixed-train variant gives the same
  spike counts as the reference's own CUDA build.
- A 24-network ensemble (ensemble.py) against the oracle neuron by neuron, and one network
  simulated alone against the same network inside the ensemble.
"""
import os

import numpy as np
import pytest

import nestgpu as ngpu
import oracle as orc
from ensemble import build_ensemble, ensemble_spec
from workloads import balanced_network, benchmark_network

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnestgpukernel.so")


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    yield
    ngpu.Reset()


def oracle_segments(conn, dt, skip_sources):
    """Oracle connections as (segment key, target, port, weight), sorted; the segment key is
    source * dspan + delay step - dmin over the recurrent edges."""
    keep = ~np.isin(conn["source"], skip_sources)
    src = conn["source"][keep].astype(np.int64)
    step = np.round(conn["delay"][keep] / np.float32(dt)).astype(np.int64) - 1
    return src, step, conn["target"][keep], conn["port"][keep], conn["weight"][keep]


@pytest.mark.parametrize("tpi,pf,occ", [(0, 0, 0), (1, 1, 1), (1, 0, 2)])
def test_benchmark_network_slice_matches_oracle(tpi, pf, occ):
    seed = 20240
    ngpu.SetUpdateTrialIter(tpi)
    ngpu.SetDeliverPrefetch(pf)
    ngpu.SetUpdateOccupancy(occ)
    ngpu.SetRk5Budget(1)
    neuron, pg = benchmark_network(ngpu, 0.01, seed)
    ngpu.Calibrate()
    csr = ngpu.GetDeliveryCsr()
    o = orc.Oracle()
    oneuron, opg = benchmark_network(o, 0.01, seed)
    src, step, tgt, port, w = oracle_segments(o.ConnectionArrays(), 0.1, [opg[0]])
    n_nodes, dmin, dspan = csr["n_nodes"], csr["dmin"], csr["dspan"]
    assert len(src) == len(neuron) * 1000 == len(csr["target"])
    assert dmin == 9 and dspan == 11          # delays 1.0 .. 2.0 ms on the 0.1 ms grid
    key = src * dspan + (step - dmin)
    assert key.min() >= 0 and key.max() < n_nodes * dspan
    # segment sizes
    cnt = np.bincount(key, minlength=n_nodes * dspan)
    assert np.array_equal(np.diff(csr["seg_off"]), cnt)
    # segment contents, as sorted (key, target, port, weight) lists
    gkey = np.repeat(np.arange(n_nodes * dspan, dtype=np.int64), np.diff(csr["seg_off"]))
    o_ord = np.lexsort((w, port, tgt, key))
    g_ord = np.lexsort((csr["weight"], csr["port"], csr["target"], gkey))
    assert np.array_equal(key[o_ord], gkey[g_ord])
    assert np.array_equal(tgt[o_ord], csr["target"][g_ord])
    assert np.array_equal(port[o_ord], csr["port"][g_ord].astype(np.int32))
    assert np.array_equal(w[o_ord], csr["weight"][g_ord])
    # in-degree 800 exc (port 0) + 200 inh (port 1) per neuron; sources in range
    deg = np.bincount(tgt * 2 + port, minlength=2 * (len(neuron) + 1)).reshape(-1, 2)
    deg = deg[neuron.i0:neuron.i0 + len(neuron)]
    assert (deg[:, 0] == 800).all() and (deg[:, 1] == 200).all()
    # 200 ms of simulation: spike counts, events and state bit for bit
    ngpu.Simulate(200.0)
    o.Simulate(200.0)
    c_gpu = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
    c_orc = np.asarray(o.GetStatus(oneuron, "spike_count")).ravel()
    assert c_gpu.sum() > 1000
    assert np.array_equal(c_gpu, c_orc)
    assert ngpu.GetStats()["n_events"] == o.NEvents()
    for var in ("V_m", "w"):
        a = np.float32(np.asarray(ngpu.GetStatus(neuron, var)).ravel())
        b = np.float32(np.asarray(o.GetStatus(oneuron, var)).ravel())
        assert np.array_equal(a, b), var
    assert ngpu.GetStats()["status"] == 0


def test_balanced_network_as_specified_matches_oracle():
    recorded = [0, 1, 799, 800, 999]
    res = []
    for api in (ngpu, orc.Oracle()):
        neuron = balanced_network(api, seed=42, drive="poisson")
        rec = api.CreateRecord("", ["V_m"] * len(recorded) + ["w"] * len(recorded),
                               [neuron[i] for i in recorded] * 2, [0] * (2 * len(recorded)))
        api.Simulate(1000.0)
        counts = np.asarray(api.GetStatus(neuron, "spike_count")).ravel()
        data = np.float32(np.asarray(api.GetRecordData(rec), dtype=np.float64))
        res.append((counts, data))
    (c_gpu, d_gpu), (c_orc, d_orc) = res
    assert c_gpu.sum() > 0
    assert np.array_equal(c_gpu, c_orc)
    assert d_gpu.shape == (10001, 1 + 2 * len(recorded))     # initial row + one per step
    assert np.array_equal(d_gpu, d_orc)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")
def test_balanced_network_fixed_trains_matches_reference_build():
    from test_gpu_reference import run_reference
    ref = run_reference("balanced_trains:1000")
    neuron = balanced_network(ngpu, seed=42, drive="trains", t_sim=1000.0)
    ngpu.Simulate(1000.0)
    counts = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
    o = orc.Oracle()
    oneuron = balanced_network(o, seed=42, drive="trains", t_sim=1000.0)
    o.Simulate(1000.0)
    assert counts.sum() > 0
    assert np.array_equal(counts, np.asarray(o.GetStatus(oneuron, "spike_count")).ravel())
    assert counts.tolist() == ref["counts"]


def small_spec():
    return ensemble_spec(n_networks=24, seed=5, median=1500, lo=1000, hi=4000)


def ensemble_counts(api, spec, t_ms):
    groups, layout = build_ensemble(api, spec)
    api.Simulate(t_ms)
    return {m: np.asarray(api.GetStatus(g, "spike_count")).ravel() for m, g in groups.items()}, layout


def test_ensemble_matches_oracle_neuron_by_neuron():
    spec = small_spec()
    c_gpu, layout = ensemble_counts(ngpu, spec, 200.0)
    c_orc, _ = ensemble_counts(orc.Oracle(), spec, 200.0)
    assert set(c_gpu) == {"aeif_cond_beta_multisynapse", "iaf_psc_exp"}
    for m in c_gpu:
        assert c_gpu[m].sum() > 0
        assert np.array_equal(c_gpu[m], c_orc[m]), m
    assert ngpu.GetStats()["status"] == 0


def test_network_alone_equals_network_in_ensemble():
    spec = small_spec()
    counts, layout = ensemble_counts(ngpu, spec, 200.0)
    picked = {}
    for i, (model, off, n) in enumerate(layout):
        picked.setdefault(model, i)
    assert len(picked) == 2
    for model, i in picked.items():
        _, off, n = layout[i]
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        alone, _ = ensemble_counts(ngpu, [spec[i]], 200.0)
        assert alone[model].sum() > 0
        assert np.array_equal(alone[model], counts[model][off:off + n]), model
