"""Scenarios shared by the oracle tests and the CUDA-engine parity tests.

Each function takes `api`: either the engine's `nestgpu` module or an
`oracle.Oracle` instance; both expose the reference's nestgpu.py calling
conventions.  The scenarios restate the reference's own tests
(python/test/test_<model>.py, test_connect.py, test_brunel_list.py) and add
seeded networks for bit-exact comparisons.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_traces():
    return np.load(os.path.join(GOLDEN, "nest_traces.npz"))


def trace_scenario(api, model):
    """Single neuron driven by a two-spike spike_generator through every
    receptor; returns the recorded V_m trace (mV, one row per 0.1 ms step).
    Follows python/test/test_<model>.py of the reference."""
    sg_times = [10.0, 400.0]
    if model in ("aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse"):
        neuron = api.Create(model, 1, 3)
        st = {"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
              "E_rev": [20.0, 0.0, -85.0]}
        if model == "aeif_cond_beta_multisynapse":
            st["tau_decay"] = [40.0, 20.0, 30.0]
            st["tau_rise"] = [20.0, 10.0, 5.0]
        else:
            st["tau_syn"] = [40.0, 20.0, 30.0]
        api.SetStatus(neuron, st)
        delay = [1.0, 100.0, 130.0]
        weight = [0.1, 0.2, 0.5]
        var = "V_m"
    elif model in ("aeif_psc_exp_multisynapse", "aeif_psc_alpha_multisynapse"):
        neuron = api.Create(model, 1, 2)
        api.SetStatus(neuron, {"V_peak": 0.0, "a": 4.0, "b": 80.5, "E_L": -70.6, "g_L": 300.0,
                               "tau_syn": [40.0, 20.0]})
        delay = [1.0, 100.0]
        weight = [1.0, -2.0]
        var = "V_m"
    elif model == "iaf_psc_exp":
        neuron = api.Create("iaf_psc_exp")
        delay = [1.0, 100.0]
        weight = [1.0, -2.0]
        var = "V_m_rel"
    else:
        raise ValueError(model)
    spike = api.Create("spike_generator")
    api.SetStatus(spike, {"spike_times": sg_times})
    for syn in range(len(delay)):
        api.Connect(spike, neuron, {"rule": "all_to_all"},
                    {"receptor": syn, "weight": weight[syn], "delay": delay[syn]})
    rec = api.CreateRecord("", [var], [neuron[0]], [0])
    api.Simulate(800.0)
    data = np.asarray(api.GetRecordData(rec), dtype=np.float64)
    v = data[:, 1]
    if model == "iaf_psc_exp":
        v = -70.0 + v
    return data[:, 0], v


def trace_rmse(v, ref):
    """The reference tests' metric: std of the difference at 1 ms sampling,
    relative to |mean V_m| (python/test/test_aeif_cond_beta_multisynapse.py:45-50)."""
    dv = np.array([v[i * 10 + 20] - ref[i, 1] for i in range(len(ref))])
    return float(np.std(dv) / abs(np.mean(v)))


def connect_scenario(api):
    """python/test/test_connect.py: all_to_all with weight/delay arrays between even and
    odd neurons; returns {section: [status dict | [weight, delay]]}."""
    N = 5
    neuron = api.Create("aeif_cond_beta_multisynapse", 2 * N)
    even = [neuron[2 * i] for i in range(N)]
    odd = [neuron[2 * i + 1] for i in range(N)]
    e2o_d, e2o_w, o2e_d, o2e_w = [], [], [], []
    for itgt in range(N):
        ite, ito = 2 * itgt, 2 * itgt + 1
        for isrc in range(N):
            ise, iso = 2 * isrc, 2 * isrc + 1
            e2o_d.append(2.0 * N * ise + ito)
            e2o_w.append(100.0 * (2.0 * N * ise + ito))
            o2e_d.append(2.0 * N * iso + ite)
            o2e_w.append(100.0 * (2.0 * N * iso + ite))
    api.Connect(even, odd, {"rule": "all_to_all"}, {"weight_array": e2o_w, "delay_array": e2o_d})
    api.Connect(odd, even, {"rule": "all_to_all"}, {"weight_array": o2e_w, "delay_array": o2e_d})
    out = {}
    status = getattr(api, "GetConnStatusList", None)

    def st(ids, key=None):
        if status is not None:
            return status(ids, key)
        return api.GetStatus(ids, key)

    ids = api.GetConnections(even, neuron)
    out["Even to all"] = st(ids)
    out["Even to all weight, delat"] = st(ids, ["weight", "delay"])
    out["All to odd"] = st(api.GetConnections(neuron, odd))
    n36 = neuron[3:7]
    out["Even to 3,4,5,6"] = st(api.GetConnections(even, n36))
    out["3,4,5,6 to odd"] = st(api.GetConnections(n36, odd))
    return out


def fixed_train_network(api, n=60, n_in=20, seed=7, t_sim=300.0, model="aeif_cond_beta_multisynapse",
                        record=True):
    """Recurrent network driven by fixed spike_generator trains (no Poisson), for
    bit-exact spike counts.  Connectivity comes from the engine's own RandomInt
    stream (fixed_indegree / fixed_total_number with normal_clipped delays)."""
    rng = np.random.RandomState(seed)
    api.SetKernelStatus("rnd_seed", 1000 + seed)
    if model == "iaf_psc_exp":
        neuron = api.Create("iaf_psc_exp", n)
        api.SetStatus(neuron, {"I_e": 370.0})
        w_exc, w_inh, w_in = 35.0, -60.0, 90.0
        rec_var = "V_m_rel"
    elif model in ("aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse"):
        neuron = api.Create(model, n, 2)
        api.SetStatus(neuron, {"E_rev": [0.0, -85.0], "I_e": 500.0})
        w_exc, w_inh, w_in = 2.0, 4.0, 6.0
        rec_var = "V_m"
    else:
        # current-based aeif: inhibition through a negative weight on receptor 1
        neuron = api.Create(model, n, 2)
        api.SetStatus(neuron, {"I_e": 500.0, "tau_syn": [2.0, 5.0]})
        w_exc, w_inh, w_in = 60.0, -120.0, 200.0
        rec_var = "V_m"
    n_exc = int(0.8 * n)
    exc = neuron[0:n_exc]
    inh = neuron[n_exc:n]
    gens = api.Create("spike_generator", n_in)
    for i in range(n_in):
        t = np.cumsum(rng.exponential(8.0, size=64)) + 1.0
        t = np.round(t[t < t_sim - 1.0], 1)
        t = np.unique(t)
        api.SetStatus([gens[i]], {"spike_times": [float(x) for x in t]})
    api.Connect(exc, neuron, {"rule": "fixed_indegree", "indegree": 10},
                {"weight": w_exc, "receptor": 0,
                 "delay": {"distribution": "normal_clipped", "mu": 1.5, "low": 0.5, "high": 3.0,
                           "sigma": 0.6}})
    inh_port = 1
    api.Connect(inh, neuron, {"rule": "fixed_total_number", "total_num": 4 * n},
                {"weight": w_inh, "receptor": inh_port, "delay": 0.8})
    api.Connect(gens, neuron, {"rule": "fixed_indegree", "indegree": 3},
                {"weight": w_in, "receptor": 0, "delay": 1.0})
    api.ActivateSpikeCount(neuron)
    rec = None
    if record:
        rec = api.CreateRecord("", [rec_var] * 3 + ["spike"] * 2, [neuron[0], neuron[1], neuron[n - 1],
                                                                  neuron[0], neuron[5]], [0] * 5)
    api.Simulate(t_sim)
    counts = np.asarray(api.GetStatus(neuron, "spike_count")).ravel().astype(np.int64)
    data = np.asarray(api.GetRecordData(rec)) if record else None
    return counts, data


def many_port_network(api, model, nport, n=40, n_in=12, seed=11, t_sim=150.0):
    """aeif neurons with `nport` receptors (1 up to the reference's maximum of 20), each port
    with its own time constants (and reversal potential for the conductance models), driven by
    fixed spike_generator trains spread over all ports plus recurrent connections onto the
    last port. Returns spike counts and a record of V_m and the input variable of the first
    and the last port."""
    rng = np.random.RandomState(seed)
    api.SetKernelStatus("rnd_seed", 2000 + seed)
    neuron = api.Create(model, n, nport)
    taus = [float(x) for x in np.round(np.linspace(1.0, 12.0, nport), 3)]
    if model == "aeif_cond_beta_multisynapse":
        api.SetStatus(neuron, {"E_rev": [-85.0 if p % 3 == 2 else 0.0 for p in range(nport)],
                               "tau_rise": [0.2 + 0.1 * (p % 5) for p in range(nport)],
                               "tau_decay": taus, "I_e": 650.0})
        w, w_rec, var = 3.0, 1.5, "g"
    elif model == "aeif_cond_alpha_multisynapse":
        api.SetStatus(neuron, {"E_rev": [-85.0 if p % 3 == 2 else 0.0 for p in range(nport)],
                               "tau_syn": taus, "I_e": 650.0})
        w, w_rec, var = 1.0, 0.5, "g"
    else:
        api.SetStatus(neuron, {"tau_syn": taus, "I_e": 650.0})
        w, w_rec, var = (150.0, 80.0, "I_syn") if model == "aeif_psc_exp_multisynapse" else (50.0, 30.0, "I_syn")
    gens = api.Create("spike_generator", n_in)
    for i in range(n_in):
        t = np.cumsum(rng.exponential(6.0, size=48)) + 1.0
        t = np.unique(np.round(t[t < t_sim - 1.0], 1))
        api.SetStatus([gens[i]], {"spike_times": [float(x) for x in t]})
    for p in range(nport):
        sign = -1.0 if (model not in ("aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse")
                        and p % 3 == 2) else 1.0
        api.Connect(gens, neuron, {"rule": "fixed_indegree", "indegree": max(2, n_in // nport)},
                    {"weight": sign * w, "receptor": p, "delay": 1.0 + 0.1 * (p % 4)})
    api.Connect(neuron, neuron, {"rule": "fixed_total_number", "total_num": 3 * n},
                {"weight": w_rec, "receptor": nport - 1, "delay": 1.2})
    api.ActivateSpikeCount(neuron)
    rec = api.CreateRecord("", ["V_m", var, var], [neuron[0], neuron[1], neuron[2]], [0, 0, nport - 1])
    api.Simulate(t_sim)
    counts = np.asarray(api.GetStatus(neuron, "spike_count")).ravel().astype(np.int64)
    return counts, np.asarray(api.GetRecordData(rec))


def poisson_network(api, n=200, rate=12000.0, t_sim=200.0, seed=3, model="aeif_cond_beta_multisynapse"):
    """Neurons driven only by one poisson_generator (all_to_all) plus sparse recurrent
    coupling; used for bit-exact comparison of the counter-based Poisson drive."""
    api.SetKernelStatus("rnd_seed", seed)
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", rate)
    if model == "iaf_psc_exp":
        neuron = api.Create("iaf_psc_exp", n)
        w = 60.0
    else:
        neuron = api.Create(model, n, 2)
        api.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
        w = 0.4
    api.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": w, "delay": 0.2, "receptor": 0})
    api.Connect(neuron, neuron, {"rule": "fixed_total_number", "total_num": 8 * n},
                {"weight": w * 0.5, "delay": 1.3, "receptor": 0})
    api.ActivateSpikeCount(neuron)
    api.Simulate(t_sim)
    return np.asarray(api.GetStatus(neuron, "spike_count")).ravel().astype(np.int64)



from workloads import c4_network  # noqa: E402,F401  (shared with bench.py)


def _conn_status(api, ids, key):
    status = getattr(api, "GetConnStatusList", None)
    return status(ids, key) if status is not None else api.GetStatus(ids, key)


def stdp_expected(w, Dt, tau_plus, tau_minus, lambd, alpha, mu_plus, mu_minus, Wmax):
    """The weight after one pre/post pair at Dt = t_post - t_pre (ms), as the reference's
    python/test/test_stdp.py states it (Guetig et al. 2003, step size lambda * Wmax)."""
    if Dt >= 0:
        w1 = w + lambd * Wmax * np.exp(-Dt / tau_plus) * (1.0 - w / Wmax) ** mu_plus
        return min(w1, Wmax)
    w1 = w - alpha * lambd * Wmax * np.exp(Dt / tau_minus) * (w / Wmax) ** mu_minus
    return max(w1, 0.0)


STDP_PAR = {"tau_plus": 20.0, "tau_minus": 20.0, "lambda": 1.0, "alpha": 1.0, "mu_plus": 1.0,
            "mu_minus": 1.0, "Wmax": 0.001}


def stdp_pair_scenario(api, n=50, dt_step=5.0, par=None, model="aeif_cond_beta_multisynapse"):
    """python/test/test_stdp.py: n presynaptic/postsynaptic pairs, each neuron driven once by a
    strong spike_generator input so that it spikes once; the plastic edge pre[i] -> post[i] has
    a delay making the post spike follow the pre spike's arrival by Dt_i = dt_step*(i-(n-1)/2)
    ms (negative: depression, positive: potentiation).  Returns (Dt list, simulated weights,
    expected weights)."""
    par = dict(STDP_PAR if par is None else par)
    syn = api.CreateSynGroup("stdp", par)
    sg = api.Create("spike_generator", n)
    neuron = api.Create(model, 2 * n)
    api.SetStatus(neuron, {"t_ref": 1000.0})
    pre, post = neuron[0:n], neuron[n:2 * n]
    dts = [dt_step * (i - 0.5 * (n - 1)) for i in range(n)]
    api.SetStatus(sg, {"spike_times": [50.0], "spike_heights": [1.0]})
    time_diff, delay0, w_sg = 400.0, 1.0, 17.9
    w0 = par["Wmax"] / 2
    api.Connect(sg, pre, {"rule": "one_to_one"}, {"weight": w_sg, "delay": delay0})
    api.Connect(sg, post, {"rule": "one_to_one"}, {"weight": w_sg, "delay": delay0 + time_diff})
    for i in range(n):
        api.Connect([pre[i]], [post[i]], {"rule": "one_to_one"},
                    {"weight": w0, "delay": time_diff - dts[i], "synapse_group": syn})
    api.Simulate(1000.0)
    ids = api.GetConnections(pre, post)
    w = np.asarray(_conn_status(api, ids, "weight"), dtype=np.float64)
    exp = [stdp_expected(w0, d, par["tau_plus"], par["tau_minus"], par["lambda"], par["alpha"],
                         par["mu_plus"], par["mu_minus"], par["Wmax"]) for d in dts]
    return dts, w, np.asarray(exp)


def plastic_network(api, n=80, n_in=20, seed=11, t_sim=400.0, model="aeif_cond_beta_multisynapse"):
    """A recurrent network with plastic excitatory edges (STDP group) and static inhibitory
    ones, driven by fixed spike_generator trains (no Poisson): spike counts and the final
    plastic weights are deterministic.  Returns (spike counts, plastic weights in connection
    order)."""
    rng = np.random.RandomState(seed)
    api.SetKernelStatus("rnd_seed", 2000 + seed)
    stdp = {"tau_plus": 20.0, "tau_minus": 25.0, "lambda": 0.05, "alpha": 1.1, "mu_plus": 0.5,
            "mu_minus": 0.8}
    if model == "iaf_psc_exp":
        syn = api.CreateSynGroup("stdp", dict(stdp, Wmax=80.0))
        neuron = api.Create("iaf_psc_exp", n)
        api.SetStatus(neuron, {"I_e": 370.0})
        w_exc, w_inh, w_in = 35.0, -60.0, 90.0
    else:
        syn = api.CreateSynGroup("stdp", dict(stdp, Wmax=3.0))
        neuron = api.Create(model, n, 2)
        api.SetStatus(neuron, {"E_rev": [0.0, -85.0], "t_ref": 2.0})
        w_exc, w_inh, w_in = 1.5, 8.0, 2.0
    n_exc = int(0.8 * n)
    exc, inh = neuron[0:n_exc], neuron[n_exc:n]
    gens = api.Create("spike_generator", n_in)
    for i in range(n_in):
        t = np.cumsum(rng.exponential(6.0, size=96)) + 1.0
        t = np.unique(np.round(t[t < t_sim - 1.0], 1))
        api.SetStatus([gens[i]], {"spike_times": [float(x) for x in t]})
    api.Connect(exc, neuron, {"rule": "fixed_indegree", "indegree": 10},
                {"weight": w_exc, "receptor": 0, "synapse_group": syn,
                 "delay": {"distribution": "normal_clipped", "mu": 1.5, "low": 0.5, "high": 3.0,
                           "sigma": 0.6}})
    api.Connect(inh, neuron, {"rule": "fixed_total_number", "total_num": 4 * n},
                {"weight": w_inh, "receptor": 1, "delay": 0.8})
    api.Connect(gens, neuron, {"rule": "fixed_indegree", "indegree": 3},
                {"weight": w_in, "receptor": 0, "delay": 1.0})
    api.ActivateSpikeCount(neuron)
    api.Simulate(t_sim)
    counts = np.asarray(api.GetStatus(neuron, "spike_count")).ravel()
    ids = api.GetConnections(exc, neuron)
    w = np.asarray(_conn_status(api, ids, "weight"), dtype=np.float32)
    return counts, w


def stdp_wrap_network(api, t_sim=7000.0):
    """Plastic edges driven by regular spike trains for longer than 2^16 steps, so the 16-bit
    arrival stamps pass both reset points (time index 0x8000 and 0x10000,
    src/nestgpu.cu:490-498).  Besides four regular presynaptic neurons, one never spikes (its
    stamps keep the initial 0x8000 until the first reset) and one spikes only in the first
    200 ms (its stamps are more than 2^16 steps old at the end): without the resets their
    edges would be potentiated by the later postsynaptic spikes.  Returns the plastic weights
    in connection order (sources: the four regular neurons, the silent one, the early one)."""
    syn = api.CreateSynGroup("stdp", {"tau_plus": 20.0, "tau_minus": 20.0, "lambda": 0.002,
                                      "alpha": 1.0, "mu_plus": 1.0, "mu_minus": 1.0, "Wmax": 2.0})
    sg = api.Create("spike_generator", 5)
    pre = api.Create("iaf_psc_exp", 6)     # 0-3 regular, 4 silent, 5 early
    post = api.Create("iaf_psc_exp", 4)
    for i in range(4):
        t = np.arange(20.0 + 3.0 * i, t_sim - 10.0, 47.0 + 6.0 * i)
        api.SetStatus([sg[i]], {"spike_times": [float(round(x, 1)) for x in t]})
    api.SetStatus([sg[4]], {"spike_times": [100.0, 150.0]})
    api.Connect(sg[0:4], pre[0:4], {"rule": "one_to_one"}, {"weight": 5000.0, "delay": 1.0})
    api.Connect([sg[4]], [pre[5]], {"rule": "one_to_one"}, {"weight": 5000.0, "delay": 1.0})
    api.Connect(sg[0:4], post, {"rule": "one_to_one"}, {"weight": 5000.0, "delay": 4.0})
    api.Connect(pre, post, {"rule": "all_to_all"},
                {"weight": 1.0, "delay": {"distribution": "normal_clipped", "mu": 3.0, "sigma": 1.5,
                                          "low": 0.5, "high": 8.0}, "synapse_group": syn})
    api.Simulate(t_sim)
    ids = api.GetConnections(pre, post)
    return np.asarray(_conn_status(api, ids, "weight"), dtype=np.float32)


# The reference's STDP cases (python/test/test_stdp/cases/case1-10.py): one presynaptic and
# one postsynaptic parrot_neuron, each driven by a spike_generator (weight 1, delay 1 ms); the
# plastic edge enters the postsynaptic parrot on receptor 1 (weight 0 there, so it does not
# make it fire).  (pre spike times, post spike times, postsynaptic den_delay, plastic delay).
STDP_CASES = {
    1: ([2.0], [1.0, 3.0], 3.0, 1.0),
    2: ([4.0], [1.0, 5.0], 3.0, 1.0),
    3: ([4.0, 6.5], [1.0, 5.0, 6.0], 3.0, 1.0),
    4: ([2.0, 6.5], [1.0, 5.0, 6.0], 3.0, 1.0),
    5: ([1.0], [1.0], 3.0, 1.0),
    6: ([1.0, 3.0], [2.0], 1.0, 3.0),
    7: ([1.0, 5.0], [4.0], 1.0, 3.0),
    8: ([1.0, 5.0, 6.0], [4.0, 6.5], 1.0, 3.0),
    9: ([1.0, 5.0, 6.0], [2.0, 6.5], 1.0, 3.0),
    10: ([1.0], [1.0], 1.0, 3.0),
}
STDP_CASE_PAR = {"tau_plus": 20.0, "tau_minus": 20.0, "lambda": 0.01, "alpha": 1.0, "mu_plus": 1.0,
                 "mu_minus": 1.0, "Wmax": 10.0}


def stdp_case_expected(case, w0=1.0):
    """The weight after the case's spikes: a presynaptic spike reaches the synapse `delay`
    after it is emitted and is depressed against the last postsynaptic spike that reached
    the synapse before it; a postsynaptic spike reaches it `den_delay` after it is emitted
    and potentiates against the last presynaptic arrival at or before it (the pairing that
    the cases' closed forms follow)."""
    pre, post, den, delay = STDP_CASES[case]
    p = STDP_CASE_PAR
    ev = sorted([(t + delay, 0) for t in pre] + [(t + den, 1) for t in post], key=lambda e: (e[0], -e[1]))
    w, last_pre, last_post = w0, None, None
    for t, kind in ev:
        if kind == 0:
            if last_post is not None and t - last_post > 0:
                w = stdp_expected(w, last_post - t, p["tau_plus"], p["tau_minus"], p["lambda"], p["alpha"],
                                  p["mu_plus"], p["mu_minus"], p["Wmax"])
            last_pre = t
        else:
            if last_pre is not None:
                w = stdp_expected(w, t - last_pre, p["tau_plus"], p["tau_minus"], p["lambda"], p["alpha"],
                                  p["mu_plus"], p["mu_minus"], p["Wmax"])
            last_post = t
    return w


def stdp_case(api, case, w0=1.0, sim_time=20.0):
    """Runs one reference STDP case; returns the simulated weight of the plastic edge."""
    pre_t, post_t, den, delay = STDP_CASES[case]
    pre = api.Create("parrot_neuron")
    post = api.Create("parrot_neuron")
    sg_pre = api.Create("spike_generator")
    sg_post = api.Create("spike_generator")
    api.SetStatus(sg_pre, {"spike_times": pre_t})
    api.SetStatus(sg_post, {"spike_times": post_t})
    api.Connect(sg_pre, pre, {"rule": "one_to_one"}, {"weight": 1.0, "delay": 1.0})
    api.Connect(sg_post, post, {"rule": "one_to_one"}, {"weight": 1.0, "delay": 1.0})
    syn = api.CreateSynGroup("stdp", STDP_CASE_PAR)
    api.SetStatus(post, {"den_delay": den})
    api.Connect(pre, post, {"rule": "one_to_one"},
                {"weight": w0, "delay": delay, "synapse_group": syn, "receptor": 1})
    api.Simulate(sim_time)
    return float(_conn_status(api, api.GetConnections(pre, post), "weight")[0])


def parrot_scenario(api):
    """Parrot neurons repeating spike-generator trains on port 0 (port 1 weighted 0), one with
    hold_spike_height; returns (spike counts, recorded V columns)."""
    sg = api.Create("spike_generator", 2)
    p = api.Create("parrot_neuron", 3)
    api.SetStatus([sg[0]], {"spike_times": [2.0, 5.0, 5.3, 9.9], "spike_heights": [2.0, 3.0, 1.0, 4.0]})
    api.SetStatus([sg[1]], {"spike_times": [1.0, 4.0, 6.0]})
    api.Connect(sg, p[0:1], {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    api.Connect(sg, p[1:2], {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0, "receptor": 1})
    api.Connect(sg, p[2:3], {"rule": "all_to_all"}, {"weight": 0.5, "delay": 2.0})
    api.SetStatus(p[2:3], {"hold_spike_height": 1.0})
    api.ActivateSpikeCount(p)
    rec = api.CreateRecord("", ["V", "V", "V", "input_spike_height"], [p[0], p[1], p[2], p[2]], [0, 0, 0, 0])
    api.Simulate(15.0)
    return np.asarray(api.GetStatus(p, "spike_count")).ravel(), np.asarray(api.GetRecordData(rec))


def plastic_den_delay_network(api):
    """plastic_network's aeif variant with dendritic delays of 0, 0.5 and 2 ms on the targets."""
    orig_create = api.Create

    class WithDen(object):
        def __getattr__(self, name):
            return getattr(api, name)

        def Create(self, model, n=1, n_port=1, *args, **kw):
            nodes = orig_create(model, n, n_port, *args, **kw)
            if model == "aeif_cond_beta_multisynapse":
                for i in range(n):
                    api.SetStatus([nodes[i]], {"den_delay": [0.0, 0.5, 2.0][i % 3]})
            return nodes

    return plastic_network(WithDen())


def syn_model_scenario(api, n=5, fact=0.2, offset=0.03):
    """python/test/test_syn_model.py: pairs of neurons each firing once, the second dt_i after
    the first's spike arrives through an edge of the linear test synapse model (weight 0, so
    it changes nothing in the dynamics); the weight afterwards is dt_i * fact + offset."""
    g = api.CreateSynGroup("test_syn_model", {"fact": fact, "offset": offset})
    sg = api.Create("spike_generator", n)
    neuron = api.Create("aeif_cond_beta_multisynapse", 2 * n)
    api.SetStatus(neuron, {"t_ref": 10.0})
    n0, n1 = neuron[0:n], neuron[n:2 * n]
    dts = [0.1 * (i - 0.5 * (n - 1)) for i in range(n)]
    api.SetStatus(sg, {"spike_times": [50.0], "spike_heights": [1.0]})
    api.Connect(sg, n0, {"rule": "one_to_one"}, {"weight": 17.9, "delay": 1.0, "receptor": 0,
                                                  "synapse_group": 0})
    api.Connect(sg, n1, {"rule": "one_to_one"}, {"weight": 17.9, "delay": 11.0, "receptor": 0,
                                                  "synapse_group": 0})
    for i in range(n):
        api.Connect([n0[i]], [n1[i]], {"rule": "one_to_one"},
                    {"weight": 0.0, "delay": 10.0 - dts[i], "receptor": 0, "synapse_group": g})
    api.Simulate(200.0)
    w = np.asarray(_conn_status(api, api.GetConnections(n0, n1), "weight"), dtype=np.float64)
    return w, np.asarray([d * fact + offset for d in dts])


def spike_detector_scenario(api, n=30, t1=490.0, t2=10.0):
    """python/test/test_spike_times.py: aeif neurons driven by a Poisson generator, each
    followed one_to_one by a spike_detector (delay 0.1 ms) whose spike_height is recorded;
    returns (recorded rows, spike counts, recorded spike times)."""
    api.SetKernelStatus("rnd_seed", 1234)
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 500.0)
    neuron = api.Create("aeif_cond_beta_multisynapse", n)
    api.ActivateSpikeCount(neuron)
    api.ActivateRecSpikeTimes(neuron, 500)
    sd = api.Create("spike_detector", n)
    api.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": 4.0, "delay": 0.2})
    api.Connect(neuron, sd, {"rule": "one_to_one"}, {"weight": 1.0, "delay": 0.1})
    rec = api.CreateRecord("", ["spike_height"] * n, [sd[i] for i in range(n)], [0] * n)
    api.Simulate(t1)
    api.SetStatus(pg, "rate", 0.0)
    api.Simulate(t2)
    data = np.asarray(api.GetRecordData(rec), dtype=np.float64)
    counts = np.asarray(api.GetStatus(neuron, "spike_count")).ravel()
    times = api.GetRecSpikeTimes(neuron)
    return data, counts, times
