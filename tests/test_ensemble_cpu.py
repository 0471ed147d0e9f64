"""Ensemble specification and its construction through the engine API (no GPU work:
creation and connection calls only record the network until calibration)."""
import numpy as np

import nestgpu as ngpu
from ensemble import AEIF, IAF, build_ensemble, ensemble_spec, ensemble_synapses


def test_ensemble_spec_statistics():
    spec = ensemble_spec()
    n = np.array([s["n"] for s in spec])
    assert len(spec) == 256 and n.min() >= 1000 and n.max() <= 50000
    assert 6000 < np.median(n) < 10000
    assert sum(s["model"] == AEIF for s in spec) == round(0.6 * 256)
    k = np.array([s["indegree"] for s in spec])
    assert k.min() >= 100 and k.max() <= 500
    r = np.array([s["rate"] for s in spec])
    assert r.min() >= 5.0 and r.max() <= 20.0
    assert len(set(s["seed"] for s in spec)) == 256
    assert ensemble_synapses(spec) == int((n * k).sum())


def test_ensemble_layout_slices_groups():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    spec = ensemble_spec(n_networks=10, seed=9, median=1500, lo=1000, hi=3000)
    groups, layout = build_ensemble(ngpu, spec)
    tot = {AEIF: 0, IAF: 0}
    for net, (model, off, n) in zip(spec, layout):
        assert model == net["model"] and n == net["n"] and off == tot[model]
        tot[model] += n
    for m, g in groups.items():
        assert len(g) == tot[m]
    ngpu.Reset()


def test_network_alone_equals_network_in_ensemble_oracle():
    """Every random stream of an ensemble network is keyed by its own seed and local
    indices (generated connections, Poisson stream), so on the oracle a network simulated
    alone gives the same spikes, neuron by neuron, as inside the ensemble."""
    import oracle as orc
    spec = ensemble_spec(n_networks=6, seed=11, median=1000, lo=600, hi=1400)
    o = orc.Oracle()
    groups, layout = build_ensemble(o, spec)
    o.Simulate(100.0)
    counts = {m: np.asarray(o.GetStatus(g, "spike_count")).ravel() for m, g in groups.items()}
    assert sum(c.sum() for c in counts.values()) > 0
    for i in (0, 1, 5):
        model, off, n = layout[i]
        a = orc.Oracle()
        g1, l1 = build_ensemble(a, [spec[i]])
        a.Simulate(100.0)
        alone = np.asarray(a.GetStatus(g1[model], "spike_count")).ravel()
        assert np.array_equal(alone, counts[model][off:off + n])
