"""Batched ensemble of independent spiking networks advanced together.

Many networks of uneven size are laid out as slices of two node groups, one per
neuron model (aeif_cond_beta_multisynapse and iaf_psc_exp), with connections only
inside each network.  One simulation step then advances every network with one
update launch per model, one delivery launch and the per-network Poisson draws,
all inside the engine's captured CUDA graph; the networks' independence lives in
the data (block-diagonal connectivity, one generator per network), not in the
launches.  `nestgpu.Autotune` picks the launch mappings for the whole ensemble.

The default specification: 256 networks, sizes lognormal (median 8000, log-sd 0.8)
clipped to [1000, 50000], 60% aeif / 40% iaf_psc_exp, 80% excitatory neurons,
in-degree uniform in [100, 500] per network (80% excitatory sources), Poisson drive
of 400 inputs per neuron at a per-network rate uniform in [5, 20] Hz, delays 1.5 ms
(recurrent) and 1.0 ms (drive), per-network seeds.  Every random stream of a network
(its generated connections and its Poisson generator's stream) is keyed by the
network's own seed and network-local indices, so a network gives the same spikes
alone as inside the ensemble.
"""
import numpy as np

AEIF = "aeif_cond_beta_multisynapse"
IAF = "iaf_psc_exp"

# synaptic weights: aeif in nS (as the plain balanced network), iaf in pA (the
# microcircuit's 87.8 pA PSC amplitude, inhibition -4x)
W = {AEIF: {"exc": 0.05, "inh": 0.35, "drive": 0.1},
     IAF: {"exc": 87.8, "inh": -351.2, "drive": 87.8}}


def ensemble_spec(n_networks=256, seed=2024, median=8000, log_sd=0.8, lo=1000, hi=50000, frac_aeif=0.6):
    """Per-network model, size, in-degree, drive rate [Hz per input] and seed."""
    rng = np.random.RandomState(seed)
    sizes = np.clip(np.round(rng.lognormal(np.log(median), log_sd, n_networks)), lo, hi).astype(np.int64)
    n_aeif = int(round(frac_aeif * n_networks))
    models = np.array([AEIF] * n_aeif + [IAF] * (n_networks - n_aeif))
    models = models[rng.permutation(n_networks)]
    indeg = rng.randint(100, 501, n_networks)
    rate = rng.uniform(5.0, 20.0, n_networks)
    net_seed = rng.randint(1, 2 ** 31 - 1, n_networks)
    return [{"model": str(models[i]), "n": int(sizes[i]), "indegree": int(indeg[i]), "rate": float(rate[i]),
             "seed": int(net_seed[i])} for i in range(n_networks)]


def build_ensemble(ngpu, spec, n_inputs=400, delay=1.5, drive_delay=1.0):
    """Create the ensemble through the engine API.  Returns {model: node group} and, per
    network, (model, first index inside the model's group, size)."""
    totals = {AEIF: 0, IAF: 0}
    layout = []
    for net in spec:
        layout.append((net["model"], totals[net["model"]], net["n"]))
        totals[net["model"]] += net["n"]
    groups = {}
    if totals[AEIF]:
        groups[AEIF] = ngpu.Create(AEIF, totals[AEIF], 2)
        ngpu.SetStatus(groups[AEIF], {"E_rev": [0.0, -85.0]})
    if totals[IAF]:
        groups[IAF] = ngpu.Create(IAF, totals[IAF])
    pgs = ngpu.Create("poisson_generator", len(spec))
    for i, (net, (model, off, n)) in enumerate(zip(spec, layout)):
        g = groups[model]
        cells = g[off:off + n]
        ne = int(0.8 * n)
        exc = g[off:off + ne]
        inh = g[off + ne:off + n]
        k_exc = int(round(0.8 * net["indegree"]))
        k_inh = net["indegree"] - k_exc
        w = W[model]
        ngpu.ConnectFixedIndegreeGPU(exc, cells, k_exc, w["exc"], delay, delay, receptor=0, seed=net["seed"])
        ngpu.ConnectFixedIndegreeGPU(inh, cells, k_inh, w["inh"], delay, delay, receptor=1,
                                     seed=net["seed"] + 7919)
        ngpu.SetStatus([pgs[i]], "rate", n_inputs * net["rate"])
        # the network's Poisson input is keyed by its own seed, not by its position
        ngpu.SetPoissonStream(pgs[i:i + 1], net["seed"])
        ngpu.Connect([pgs[i]], cells, {"rule": "all_to_all"}, {"weight": w["drive"], "delay": drive_delay,
                                                               "receptor": 0})
    for g in groups.values():
        ngpu.ActivateSpikeCount(g)
    return groups, layout


def ensemble_synapses(spec):
    return int(sum(net["n"] * net["indegree"] for net in spec))


def per_network_rates(ngpu, groups, layout, counts0, t_ms):
    """Mean firing rate [Hz] of every network from the spike-count difference."""
    counts = {m: np.asarray(ngpu.GetStatus(g, "spike_count")).ravel() for m, g in groups.items()}
    out = []
    for model, off, n in layout:
        c = counts[model][off:off + n] - counts0[model][off:off + n]
        out.append(c.sum() / n / (t_ms / 1000.0))
    return np.array(out), counts
