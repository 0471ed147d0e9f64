"""Seeded synthetic workloads built through the engine's nestgpu API (or any object with
the same calling conventions, such as the CPU oracle's)."""
import numpy as np


# The 1M-neuron benchmark network: 800k exc + 200k inh aeif_cond_beta_multisynapse neurons
# with two receptors (E_rev 0 / -85 mV), 800 exc (0.05 nS, receptor 0) + 200 inh (0.35 nS,
# receptor 1) inputs per neuron drawn per target with replacement, delays uniform on the
# 0.1 ms grid in [1.0, 2.0] ms, one poisson_generator at 8 kHz into every neuron (0.1 nS,
# receptor 0, delay 1.0 ms).
BENCH_N_EXC, BENCH_N_INH = 800_000, 200_000
BENCH_K_EXC, BENCH_K_INH = 800, 200
BENCH_W_EXC, BENCH_W_INH, BENCH_W_PG = 0.05, 0.35, 0.1
BENCH_PG_RATE = 8000.0
BENCH_DELAY_MIN, BENCH_DELAY_MAX = 1.0, 2.0


def benchmark_network(api, scale=1.0, seed=20240):
    """The benchmark network at `scale` of its 1M neurons (in-degrees unchanged), built with
    the generated per-target fixed in-degree rule (ConnectFixedIndegreeGPU, seeds seed and
    seed + 7919).  Returns (neurons, generator)."""
    n_exc, n_inh = int(BENCH_N_EXC * scale), int(BENCH_N_INH * scale)
    api.SetKernelStatus("rnd_seed", seed)
    neuron = api.Create("aeif_cond_beta_multisynapse", n_exc + n_inh, 2)
    api.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
    exc, inh = neuron[0:n_exc], neuron[n_exc:n_exc + n_inh]
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", BENCH_PG_RATE)
    api.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": BENCH_W_PG, "delay": 1.0, "receptor": 0})
    api.ConnectFixedIndegreeGPU(exc, neuron, BENCH_K_EXC, BENCH_W_EXC, BENCH_DELAY_MIN, BENCH_DELAY_MAX,
                                receptor=0, seed=seed)
    api.ConnectFixedIndegreeGPU(inh, neuron, BENCH_K_INH, BENCH_W_INH, BENCH_DELAY_MIN, BENCH_DELAY_MAX,
                                receptor=1, seed=seed + 7919)
    api.ActivateSpikeCount(neuron)
    return neuron, pg


def balanced_network(api, seed=42, n=1000, drive="poisson", n_gen=400, gen_rate=10.0, t_sim=1000.0):
    """The plain small balanced network as specified: n aeif_cond_beta_multisynapse neurons
    (80% exc / 20% inh, reference default parameters, receptors E_rev 0 / -85 mV), the
    reference's fixed_indegree rule (one source draw per call, shared by all targets) with
    80 exc inputs (0.05 nS, receptor 0) and 20 inh inputs (0.35 nS, receptor 1), delay
    1.5 ms; drive on receptor 0 (0.1 nS, delay 1.0 ms):
      "poisson": n_gen poisson_generators at gen_rate Hz, all_to_all (400 x 10 Hz = 4 kHz);
      "trains":  one spike_generator per neuron, one_to_one, replaying a seeded Poisson
                 train of the same aggregate rate (n_gen x gen_rate) as spike heights per
                 0.1 ms step (deterministic input for comparisons across libraries).
    Returns the neurons."""
    api.SetKernelStatus("rnd_seed", seed)
    neuron = api.Create("aeif_cond_beta_multisynapse", n, 2)
    api.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
    ne = int(0.8 * n)
    exc, inh = neuron[0:ne], neuron[ne:n]
    api.Connect(exc, neuron, {"rule": "fixed_indegree", "indegree": 80},
                {"weight": 0.05, "delay": 1.5, "receptor": 0})
    api.Connect(inh, neuron, {"rule": "fixed_indegree", "indegree": 20},
                {"weight": 0.35, "delay": 1.5, "receptor": 1})
    if drive == "poisson":
        pg = api.Create("poisson_generator", n_gen)
        api.SetStatus(pg, "rate", gen_rate)
        api.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": 0.1, "delay": 1.0, "receptor": 0})
    elif drive == "trains":
        rng = np.random.RandomState(seed)
        lam = n_gen * gen_rate * 1e-4            # expected input spikes per 0.1 ms step
        n_steps = int(round(t_sim / 0.1))
        sg = api.Create("spike_generator", n)
        for i in range(n):
            k = rng.poisson(lam, n_steps)
            steps = np.nonzero(k)[0]
            # steps 1 .. n_steps - 1 on the 0.1 ms grid (times strictly increasing)
            steps = steps[steps > 0]
            api.SetStatus(sg[i:i + 1], {"spike_times": [round(0.1 * int(s), 1) for s in steps],
                                        "spike_heights": [float(k[s]) for s in steps]})
        api.Connect(sg, neuron, {"rule": "one_to_one"}, {"weight": 0.1, "delay": 1.0, "receptor": 0})
    else:
        raise ValueError(drive)
    api.ActivateSpikeCount(neuron)
    return neuron


def c4_network(api, seed=42, n=1000, drive_w=0.1, n_port=4):
    """The small balanced network (800 exc / 200 inh aeif_cond_beta_multisynapse,
    fixed in-degree 80 exc w=0.05 nS / 20 inh w=0.35 nS, delay 1.5 ms, 4 kHz Poisson
    drive on receptor 0) with four receptors per neuron: E_rev 0, 0, -85, -85 mV and, per
    neuron and receptor, tau_rise uniform in [0.2, 1] ms and tau_decay uniform in [2, 20] ms
    (seeded); each projection is split evenly over its two receptors.  drive_w is the
    Poisson weight (0.1 nS as in the plain network; larger values make it fire)."""
    api.SetKernelStatus("rnd_seed", seed)
    rng = np.random.RandomState(seed)
    tau_rise = np.round(rng.uniform(0.2, 1.0, (n, n_port)), 3)
    tau_decay = np.round(rng.uniform(2.0, 20.0, (n, n_port)), 3)
    neuron = api.Create("aeif_cond_beta_multisynapse", n, n_port)
    e_rev = [0.0] * (n_port // 2) + [-85.0] * (n_port - n_port // 2)
    api.SetStatus(neuron, {"E_rev": e_rev})
    for i in range(n):
        api.SetStatus(neuron[i:i + 1], {"tau_rise": [float(x) for x in tau_rise[i]],
                                        "tau_decay": [float(x) for x in tau_decay[i]]})
    ne = int(0.8 * n)
    exc, inh = neuron[0:ne], neuron[ne:n]
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 4000.0)
    half = n_port // 2
    for p in range(half):
        api.Connect(exc, neuron, {"rule": "fixed_indegree", "indegree": 80 // half},
                    {"weight": 0.05, "delay": 1.5, "receptor": p})
    for p in range(half, n_port):
        api.Connect(inh, neuron, {"rule": "fixed_indegree", "indegree": 20 // (n_port - half)},
                    {"weight": 0.35, "delay": 1.5, "receptor": p})
    api.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": drive_w, "delay": 1.0, "receptor": 0})
    api.ActivateSpikeCount(neuron)
    return neuron


# ---------------------------------------------------------------------------
# Layered cortical microcircuit (Potjans & Diesmann 2014) with iaf_psc_exp neurons,
# built the way the reference's python/Potjans_2014_s example builds it
# (network_params.py, network.py, helpers.py): 8 populations, fixed_total_number
# projections drawn from the connection-probability matrix, normal_clipped weights
# and delays, one Poisson generator per population at bg_rate x K_ext.
# ---------------------------------------------------------------------------
MC_POPS = ["L23E", "L23I", "L4E", "L4I", "L5E", "L5I", "L6E", "L6I"]
MC_N = np.array([20683, 5834, 21915, 5479, 4850, 1065, 14395, 2948])
MC_CONN_P = np.array([
    [0.1009, 0.1689, 0.0437, 0.0818, 0.0323, 0., 0.0076, 0.],
    [0.1346, 0.1371, 0.0316, 0.0515, 0.0755, 0., 0.0042, 0.],
    [0.0077, 0.0059, 0.0497, 0.135, 0.0067, 0.0003, 0.0453, 0.],
    [0.0691, 0.0029, 0.0794, 0.1597, 0.0033, 0., 0.1057, 0.],
    [0.1004, 0.0622, 0.0505, 0.0057, 0.0831, 0.3726, 0.0204, 0.],
    [0.0548, 0.0269, 0.0257, 0.0022, 0.06, 0.3158, 0.0086, 0.],
    [0.0156, 0.0066, 0.0211, 0.0166, 0.0572, 0.0197, 0.0396, 0.2252],
    [0.0364, 0.001, 0.0034, 0.0005, 0.0277, 0.008, 0.0658, 0.1443]])   # [target][source]
MC_K_EXT = np.array([1600, 1500, 2100, 1900, 2000, 1900, 2900, 2100])
MC_V0_MEAN = [-68.28, -63.16, -63.33, -63.45, -63.11, -61.66, -66.72, -61.43]
MC_V0_STD = [5.36, 4.57, 4.74, 4.94, 4.94, 4.55, 5.46, 4.48]
MC_NEURON = {"E_L": -65.0, "V_th": -50.0, "V_reset": -65.0, "C_m": 250.0, "tau_m": 10.0, "tau_syn": 0.5,
             "t_ref": 2.0}


def psc_over_psp(C_m, tau_m, tau_syn):
    """PSC amplitude (pA) that gives a 1 mV peak PSP for an exponential current."""
    sub = 1.0 / (tau_syn - tau_m)
    pre = tau_m * tau_syn / C_m * sub
    frac = (tau_m / tau_syn) ** sub
    return 1.0 / (pre * (frac ** tau_m - frac ** tau_syn))


def microcircuit_synapses(scale=1.0):
    n = np.round(MC_N * scale)
    prod = np.outer(n, n)
    with np.errstate(divide="ignore", invalid="ignore"):
        k = np.log(1.0 - MC_CONN_P) / np.log((prod - 1.0) / prod)
    return np.round(np.nan_to_num(k)).astype(np.int64)


def microcircuit(api, seed=12349, scale=1.0, dt=0.1):
    """Create and connect the microcircuit; `scale` multiplies the population sizes
    (in-degrees follow the connection probabilities).  Returns the populations."""
    nrn = MC_NEURON
    api.SetRandomSeed(seed)
    n_pop = np.round(MC_N * scale).astype(int)
    n_syn = microcircuit_synapses(scale)
    pscp = psc_over_psp(nrn["C_m"], nrn["tau_m"], nrn["tau_syn"])
    psp = np.zeros((8, 8))
    psp[:, 0::2], psp[:, 1::2] = 0.15, 0.15 * -4.0
    psp[0, 2] = 2.0 * 0.15
    w_mean = psp * pscp
    w_ext = 0.15 * pscp
    d_mean = np.zeros((8, 8))
    d_mean[:, 0::2], d_mean[:, 1::2] = 1.5, 0.75
    pops = []
    for i in range(8):
        p = api.Create("iaf_psc_exp", int(n_pop[i]))
        api.SetStatus(p, {"tau_ex": nrn["tau_syn"], "tau_in": nrn["tau_syn"], "E_L": nrn["E_L"],
                          "Theta_rel": nrn["V_th"] - nrn["E_L"], "V_reset_rel": nrn["V_reset"] - nrn["E_L"],
                          "t_ref": nrn["t_ref"], "I_e": 0.0})
        api.SetStatus(p, {"V_m_rel": {"distribution": "normal", "mu": MC_V0_MEAN[i] - nrn["E_L"],
                                      "sigma": MC_V0_STD[i]}})
        pops.append(p)
    bg = api.Create("poisson_generator", 8)
    for i in range(8):
        api.SetStatus([bg[i]], "rate", float(8.0 * MC_K_EXT[i]))
    for i, tgt in enumerate(pops):
        for j, src in enumerate(pops):
            if n_syn[i][j] <= 0:
                continue
            wm = w_mean[i][j]
            ws = abs(wm * 0.1)
            if wm < 0:
                wlo, whi, port = wm - 3.0 * ws, 0.0, 1
            else:
                wlo, whi, port = 0.0, wm + 3.0 * ws, 0
            dm = d_mean[i][j]
            ds = dm * 0.5
            api.Connect(src, tgt, {"rule": "fixed_total_number", "total_num": int(n_syn[i][j])},
                        {"weight": {"distribution": "normal_clipped", "mu": wm, "low": wlo, "high": whi,
                                    "sigma": ws},
                         "delay": {"distribution": "normal_clipped", "mu": dm, "low": dt, "high": dm + 3.0 * ds,
                                   "sigma": ds},
                         "receptor": port})
    for i, tgt in enumerate(pops):
        api.Connect([bg[i]], tgt, {"rule": "all_to_all"}, {"weight": w_ext, "delay": 1.5})
    for p in pops:
        api.ActivateSpikeCount(p)
    return pops


# ---------------------------------------------------------------------------
# Learned RK5 step proposal against the plain controller
# ---------------------------------------------------------------------------
SAFETY_INDEX = 1463   # position of the safety factor in the step model's parameter vector


def learned_vs_plain(ngpu, drive_w, log_ms=2000.0, eval_ms=1000.0, target_tuples=50_000_000,
                     max_log_ms=40000.0):
    """RK5 derivative evaluations per neuron-ms with and without the learned step proposal
    on the four-receptor balanced network: log the plain integrator on the training seed (42)
    in chunks of log_ms until target_tuples accepted steps are logged (or max_log_ms), train
    the network on the GPU, pick the safety factor on the training network, evaluate on a
    held-out seed (43), and measure there the floor: the evaluations when every step starts
    from the largest step that passes the error test (no proposal can need fewer)."""
    import time

    def evals(seed, model, t_ms, bound=False):
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        n = c4_network(ngpu, seed, drive_w=drive_w)
        ngpu.Simulate(100.0)
        if bound:
            ngpu.StepBoundMode(True)
        if model is not None:
            ngpu.StepModelSet(model)
            ngpu.StepModelEnable(True)
        nd0 = ngpu.GetStats()["n_derivs"]
        c0 = np.asarray(ngpu.GetStatus(n, "spike_count")).ravel()
        ngpu.Simulate(t_ms)
        nd1 = ngpu.GetStats()["n_derivs"]
        c1 = np.asarray(ngpu.GetStatus(n, "spike_count")).ravel()
        return (nd1 - nd0) / (len(n) * t_ms), float((c1 - c0).sum()) / len(n) / (t_ms / 1000.0)

    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    c4_network(ngpu, 42, drive_w=drive_w)
    ngpu.Simulate(100.0)
    ngpu.Rk5LogStart(target_tuples)
    t_log = 0.0
    while True:
        ngpu.Simulate(log_ms)
        t_log += log_ms
        n_log, _ = ngpu.Rk5LogCount()
        if n_log >= target_tuples or t_log >= max_log_ms:
            break
    ngpu.Rk5LogStop()
    out = {"drive_nS": drive_w, "logged_steps": n_log, "logged_bio_ms": t_log}
    t0 = time.time()
    try:
        used, loss = ngpu.StepModelTrain(iters=3000, batch=4096, lr=2e-3, safety=0.9, floor=0.0, seed=3)
        model = ngpu.StepModelGet()
    except ValueError as e:
        # no step of the plain integrator was limited by accuracy: the network would never
        # be consulted, and the learned method is the plain one
        used, model, note = 0, None, "not trained: " + str(e)
    train_s = time.time() - t0
    plain, rate_p = evals(43, None, eval_ms)
    floor, _ = evals(43, None, eval_ms, bound=True)
    out.update(plain_evals_per_neuron_ms=plain, plain_rate_hz=rate_p, floor_evals_per_neuron_ms=floor,
               largest_possible_reduction=plain / floor)
    if model is None:
        out.update(trained_on=0, learned_evals_per_neuron_ms=plain, learned_rate_hz=rate_p, ratio=1.0, note=note)
        return out
    best = None
    for sf in (0.5, 0.6, 0.7, 0.8, 0.9):
        m = model.copy()
        m[SAFETY_INDEX] = sf
        e, _ = evals(42, m, 200.0)
        if best is None or e < best[0]:
            best = (e, sf)
    model[SAFETY_INDEX] = best[1]
    learned, rate_l = evals(43, model, eval_ms)
    out.update(trained_on=used, train_mse=loss, train_s=train_s, safety=best[1],
               learned_evals_per_neuron_ms=learned, learned_rate_hz=rate_l, ratio=plain / learned)
    return out
