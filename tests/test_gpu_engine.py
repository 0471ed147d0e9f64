"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

The engine and the oracle's FP32 mode perform the same arithmetic in the same
order (explicit fused multiply-adds, the same own exp/log, the same Philox
Poisson stream), so traces, spike counts and spike times are compared bit for
bit.  The single-neuron traces are also held to the reference tests' NEST
golden tolerances, and the FP32 traces to 1e-5 relative of the FP64 oracle.
"""
import math

import numpy as np
import pytest

import nestgpu as ngpu
import oracle as orc
from scenarios import (fixed_train_network, golden_traces, poisson_network, trace_rmse,
                       trace_scenario)

pytestmark = pytest.mark.gpu

MODELS = ["aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse",
          "aeif_psc_exp_multisynapse", "aeif_psc_alpha_multisynapse", "iaf_psc_exp"]


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    yield
    ngpu.Reset()


@pytest.mark.parametrize("model", MODELS)
def test_single_neuron_trace(model):
    g = golden_traces()
    t, v = trace_scenario(ngpu, model)
    _, v32 = trace_scenario(orc.Oracle(fp64=False), model)
    _, v64 = trace_scenario(orc.Oracle(fp64=True), model)
    assert np.array_equal(np.float32(v), np.float32(v32))
    assert trace_rmse(v, g[model]) < float(g[model + "__tolerance"])
    assert np.max(np.abs(v - v64) / np.maximum(np.abs(v64), 1.0)) < 1e-5
    assert len(t) == 8001 and abs(t[-1] - 800.0) < 1e-3


@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "aeif_psc_alpha_multisynapse",
                                   "iaf_psc_exp"])
def test_recurrent_network_fixed_trains_bitexact(model):
    ngpu.SetHostRng(True)
    c_gpu, d_gpu = fixed_train_network(ngpu, model=model)
    c_orc, d_orc = fixed_train_network(orc.Oracle(), model=model)
    assert c_gpu.sum() > 0
    assert np.array_equal(c_gpu, c_orc)
    assert np.array_equal(np.float32(d_gpu), np.float32(d_orc))
    st = ngpu.GetStats()
    assert st["status"] == 0
    assert st["n_spikes"] >= c_gpu.sum()


@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "iaf_psc_exp"])
def test_poisson_driven_network_bitexact(model):
    c_gpu = poisson_network(ngpu, model=model)
    c_orc = poisson_network(orc.Oracle(), model=model)
    assert c_gpu.sum() > 100
    assert np.array_equal(c_gpu, c_orc)


def _continuation(api, chunks):
    api.SetKernelStatus("rnd_seed", 5)
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 9000.0)
    n = api.Create("aeif_cond_beta_multisynapse", 50, 2)
    api.SetStatus(n, {"E_rev": [0.0, -85.0], "t_ref": 1.0})
    api.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 0.5, "delay": 0.5})
    api.Connect(n, n, {"rule": "fixed_total_number", "total_num": 400}, {"weight": 0.3, "delay": 1.1})
    api.ActivateSpikeCount(n)
    for c in chunks:
        api.Simulate(c)
    return (np.asarray(api.GetStatus(n, "spike_count")).ravel(), np.float32(api.GetStatus(n, "V_m")),
            np.float32(api.GetStatus(n, "g1")))


def test_simulate_in_chunks_equals_one_call():
    a = _continuation(ngpu, [60.0])
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    b = _continuation(ngpu, [20.0, 25.0, 15.0])
    o = _continuation(orc.Oracle(), [20.0, 25.0, 15.0])
    for x, y, z in zip(a, b, o):
        assert np.array_equal(x, y)
        assert np.array_equal(y, z)


def test_simulation_step_api_matches_simulate():
    ngpu.SetKernelStatus("rnd_seed", 11)
    sg = ngpu.Create("spike_generator")
    ngpu.SetStatus(sg, {"spike_times": [0.3, 0.7, 1.2, 2.0]})
    n = ngpu.Create("iaf_psc_exp", 3)
    ngpu.Connect(sg, n, {"rule": "all_to_all"}, {"weight": 400.0, "delay": 0.2})
    ngpu.SetSimTime(3.0)
    ngpu.StartSimulation()
    v = []
    for _ in range(30):
        ngpu.SimulationStep()
        v.append(ngpu.GetStatus(n[0], "I_syn_ex"))
    ngpu.EndSimulation()
    o = orc.Oracle()
    sg2 = o.Create("spike_generator")
    o.SetStatus(sg2, {"spike_times": [0.3, 0.7, 1.2, 2.0]})
    n2 = o.Create("iaf_psc_exp", 3)
    o.Connect(sg2, n2, {"rule": "all_to_all"}, {"weight": 400.0, "delay": 0.2})
    o.CreateRecord("", ["I_syn_ex"], [n2[0]], [0])
    o.Simulate(3.0)
    # after a step the engine has folded that step's input, the record row has not
    assert np.float32(v[-1]) == np.float32(o.GetStatus(n2[0], "I_syn_ex")[0])
    assert max(v) > 0.0


def _step_param_changes(api, stepwise):
    """A Poisson rate and the I_e of an aeif and an iaf group changed between steps of
    a StartSimulation / SimulationStep loop (stepwise) or between Simulate calls."""
    api.SetKernelStatus("rnd_seed", 31)
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 3000.0)
    a = api.Create("aeif_cond_beta_multisynapse", 40, 2)
    api.SetStatus(a, {"E_rev": [0.0, -85.0]})
    b = api.Create("iaf_psc_exp", 20)
    api.Connect(pg, a, {"rule": "all_to_all"}, {"weight": 0.5, "delay": 1.0, "receptor": 0})
    api.Connect(pg, b, {"rule": "all_to_all"}, {"weight": 30.0, "delay": 1.0})
    api.ActivateSpikeCount(a)
    api.ActivateSpikeCount(b)
    phases = [(300, None), (300, (9000.0, 400.0, 300.0)), (300, (0.0, 0.0, 0.0))]
    out = []
    if stepwise:
        api.SetSimTime(90.0)
        api.StartSimulation()
    for k, change in phases:
        if change is not None:
            api.SetStatus(pg, "rate", change[0])
            api.SetStatus(a, "I_e", change[1])
            api.SetStatus(b, "I_e", change[2])
        if stepwise:
            for _ in range(k):
                api.SimulationStep()
        else:
            api.Simulate(k * 0.1)
        out.append(np.concatenate([np.asarray(api.GetStatus(a, "spike_count")).ravel(),
                                   np.asarray(api.GetStatus(b, "spike_count")).ravel()]))
    if stepwise:
        api.EndSimulation()
    return out


def test_parameter_changes_between_simulation_steps():
    """Parameters set between SimulationStep calls apply from the next step, as the
    reference's setters write to the device at once: the same spikes as setting them
    between Simulate calls on the oracle."""
    got = _step_param_changes(ngpu, True)
    ref = _step_param_changes(orc.Oracle(), False)
    for x, y in zip(got, ref):
        assert np.array_equal(x, y)
    # each change shows: more spikes in phase 2 than in phase 1, none added in phase 3
    d1, d2, d3 = got[0].sum(), got[1].sum() - got[0].sum(), got[2].sum() - got[1].sum()
    assert d2 > d1 and d3 < d2


def test_status_after_simulate_matches_oracle():
    def run(api):
        api.SetKernelStatus("rnd_seed", 21)
        pg = api.Create("poisson_generator")
        api.SetStatus(pg, "rate", 15000.0)
        n = api.Create("aeif_cond_beta_multisynapse", 30, 2)
        api.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 0.4, "delay": 0.3, "receptor": 1})
        api.Simulate(37.0)
        return [np.float32(api.GetStatus(n, k)) for k in ("V_m", "w", "g", "g1", "refractory_step")]
    for a, b in zip(run(ngpu), run(orc.Oracle())):
        assert np.array_equal(a, b)


def test_rec_spike_times_and_spike_record():
    def run(api):
        api.SetKernelStatus("rnd_seed", 3)
        pg = api.Create("poisson_generator")
        api.SetStatus(pg, "rate", 500.0)
        n = api.Create("aeif_cond_beta_multisynapse", 30)
        api.ActivateSpikeCount(n)
        api.ActivateRecSpikeTimes(n, 500)
        api.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 4.0, "delay": 0.2})
        api.Connect(n, n[0:1], {"rule": "all_to_all"}, {"weight": 0.01, "delay": 0.2})
        rec = api.CreateRecord("", ["spike"] * 3, [n[0], n[1], n[2]], [0, 0, 0])
        api.Simulate(490.0)
        api.SetStatus(pg, "rate", 0.0)
        api.Simulate(10.0)
        return (np.asarray(api.GetStatus(n, "spike_count")).ravel(), api.GetRecSpikeTimes(n),
                np.asarray(api.GetRecordData(rec)))
    cg, tg, rg = run(ngpu)
    co, to, ro = run(orc.Oracle())
    assert cg.sum() > 30
    assert np.array_equal(cg, co)
    assert [len(x) for x in tg] == list(cg)
    for a, b in zip(tg, to):
        assert np.array_equal(np.float32(a), np.float32(b))
    assert np.array_equal(np.float32(rg), np.float32(ro))
    # every neuron projects to neuron 0, so "spike" records each of their spikes
    assert rg[:, 1].sum() == cg[0] and rg[:, 2].sum() == cg[1] and rg[:, 3].sum() == cg[2]


def test_brunel_rate_statistics():
    """python/test/test_brunel_list.py: mean rate of 1000 aeif neurons within
    3 sqrt(rate) of 30.78 spikes/s."""
    order, n_rec = 200, 100
    ngpu.SetKernelStatus("rnd_seed", 1234)
    NE, NI = 4 * order, order
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", 20000.0)
    neuron = ngpu.Create("aeif_cond_beta_multisynapse", NE + NI, 2)
    exc, inh = neuron[0:NE], neuron[NE:NE + NI]
    ngpu.SetStatus(neuron, {"E_rev": [0.0, -85.0], "tau_decay": [1.0, 1.0], "tau_rise": [1.0, 1.0]})
    dly = {"distribution": "normal_clipped", "mu": 0.5, "low": 0.1, "high": 0.5 + 3 * 0.25, "sigma": 0.25}
    ngpu.Connect(exc, neuron.ToList(), {"rule": "fixed_indegree", "indegree": 800},
                 {"weight": 0.05, "delay": dly, "receptor": 0})
    ngpu.Connect(inh.ToList(), exc.ToList(), {"rule": "fixed_indegree", "indegree": 200},
                 {"weight": 0.35, "delay": dly, "receptor": 1})
    ngpu.Connect(inh.ToList(), inh, {"rule": "fixed_indegree", "indegree": 200},
                 {"weight": 0.35, "delay": dly, "receptor": 1})
    ngpu.Connect(pg.ToList(), neuron.ToList(), {"rule": "all_to_all"},
                 {"weight": 0.37, "delay": 0.2, "receptor": 0})
    ngpu.ActivateSpikeCount(neuron)
    ngpu.Simulate(1000.0)
    counts = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
    expected = 30.78
    rng = np.random.RandomState(0)
    sample = counts[rng.choice(NE + NI, n_rec, replace=False)]
    assert sample.min() >= expected - 3.0 * math.sqrt(expected)
    assert sample.max() <= expected + 3.0 * math.sqrt(expected)
    assert abs(sample.mean() - expected) < 3.0 * math.sqrt(expected) / math.sqrt(n_rec)
    assert len(ngpu.GetConnections(neuron[1], neuron)) == NE + NI


def test_device_rng_matches_reference_generator_for_ints():
    ngpu.SetRandomSeed(1234)
    a = np.array(ngpu.RandomInt(4096), dtype=np.uint32)
    o = orc.Oracle()
    o.SetRandomSeed(1234)
    assert np.array_equal(a, o.RandomInt(4096))


@pytest.mark.parametrize("batch_max,budget,tpi", [(1, 0, 0), (1, 2, 0), (32, 0, 0), (32, 1, 0), (3, 4, 0),
                                                  (1, 2, 1), (32, 1, 1), (32, 0, 1)])
def test_time_batching_and_straggler_handoff_keep_results(batch_max, budget, tpi):
    """Integrating several steps per kernel (up to the minimum delay) and handing long RK5
    sequences to the straggler kernel are scheduling choices: spike counts and recorded
    traces equal the oracle's for every setting."""
    ngpu.SetHostRng(True)
    ngpu.SetBatchMax(batch_max)
    ngpu.SetRk5Budget(budget)
    ngpu.SetUpdateTrialIter(tpi)
    c_gpu, d_gpu = fixed_train_network(ngpu, model="aeif_cond_beta_multisynapse", t_sim=150.0)
    c_orc, d_orc = fixed_train_network(orc.Oracle(), model="aeif_cond_beta_multisynapse", t_sim=150.0)
    assert np.array_equal(c_gpu, c_orc)
    assert np.array_equal(np.float32(d_gpu), np.float32(d_orc))


def test_profile_and_launch_counters():
    ngpu.SetHostRng(True)
    fixed_train_network(ngpu, t_sim=20.0, record=False)
    l0 = ngpu.GetLaunchCount()
    upd, rec, dlv = ngpu.ProfileSteps(50)
    assert upd > 0.0 and dlv > 0.0 and rec == 0.0
    assert ngpu.GetLaunchCount() > l0
    assert ngpu.GetStats()["steps"] == 250


@pytest.mark.parametrize("threads,group,occ,tpi,agg,pf", [(64, 8, 0, 0, 0, 0), (256, 16, 1, 0, 0, 1),
                                                          (128, 32, 1, 0, 0, 0), (64, 8, 0, 1, 0, 1),
                                                          (128, 32, 1, 1, 1, 1), (64, 32, 0, 0, 1, 0),
                                                          (128, 32, 2, 1, 0, 0), (256, 16, 2, 1, 0, 1)])
def test_launch_mappings_keep_results(threads, group, occ, tpi, agg, pf):
    """The update block size and kernel variants (register cap, one RK5 trial per loop
    iteration), the delivery lane group, warp-aggregated and pipelined delivery change only the
    launch mapping."""
    ngpu.SetHostRng(True)
    ngpu.SetUpdateThreads(threads)
    ngpu.SetDeliverGroup(group)
    ngpu.SetUpdateOccupancy(occ)
    ngpu.SetUpdateTrialIter(tpi)
    ngpu.SetDeliverAggregate(agg)
    ngpu.SetDeliverPrefetch(pf)
    c_gpu, d_gpu = fixed_train_network(ngpu, model="aeif_cond_beta_multisynapse")
    c_orc, d_orc = fixed_train_network(orc.Oracle(), model="aeif_cond_beta_multisynapse")
    assert c_gpu.sum() > 0
    assert np.array_equal(c_gpu, c_orc)
    assert np.array_equal(np.float32(d_gpu), np.float32(d_orc))


@pytest.mark.parametrize("push", [True, False])
def test_microcircuit_slice_bitexact(push):
    """The layered microcircuit at 3% size (eight iaf_psc_exp populations served by one
    multi-group launch, fixed_total_number projections with normal_clipped weights and
    delays, Poisson background): spike counts neuron by neuron equal the oracle's, with
    delivery at emission and with the delivery kernel."""
    from workloads import microcircuit
    ngpu.SetHostRng(True)
    ngpu.SetDeliverPush(push)
    pops_g = microcircuit(ngpu, scale=0.03)
    o = orc.Oracle()
    pops_o = microcircuit(o, scale=0.03)
    ngpu.Simulate(150.0)
    o.Simulate(150.0)
    c_g = np.concatenate([np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops_g])
    c_o = np.concatenate([np.asarray(o.GetStatus(p, "spike_count")).ravel() for p in pops_o])
    assert c_g.sum() > 1000
    assert np.array_equal(c_g, c_o)
    assert ngpu.DeliverPushActive() == push


def iaf_two_populations(api, seed=3, delay=1.5):
    """800 + 200 iaf_psc_exp neurons, fixed in-degree 80 + 20 with one delay, Poisson drive
    (the minimum delay sets the time batch: 1.5 ms gives 15-step batches)."""
    api.SetKernelStatus("rnd_seed", seed)
    n = api.Create("iaf_psc_exp", 1000)
    exc, inh = n[0:800], n[800:1000]
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 12000.0)
    api.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 30.0, "delay": 0.1})
    api.Connect(exc, n, {"rule": "fixed_indegree", "indegree": 80}, {"weight": 25.0, "delay": delay})
    api.Connect(inh, n, {"rule": "fixed_indegree", "indegree": 20}, {"weight": -120.0, "delay": delay})
    api.ActivateSpikeCount(n)
    return n


@pytest.mark.parametrize("delay", [0.1, 1.5])
def test_delivery_at_emission_equals_delivery_kernel(delay):
    """Delivery at emission (the update kernel's warps add each spike's out-edges into a ring of
    accumulator slots) against the delivery kernel, with one-step batches (delay 0.1 ms) and
    15-step batches (1.5 ms): the same spikes and recorded traces; events are counted when a
    spike is emitted, so at the end of a run the count also holds those still on their way
    (at most one delay's worth); the switch is refused after calibration."""
    res = []
    for push in (True, False):
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        ngpu.SetHostRng(True)
        ngpu.SetDeliverPush(push)
        n = iaf_two_populations(ngpu, delay=delay)
        rec = ngpu.CreateRecord("", ["V_m_rel", "I_syn_ex", "I_syn_in"], [n[3], n[500], n[900]], [0, 0, 0])
        ngpu.Simulate(70.0)
        ngpu.Simulate(33.0)
        assert ngpu.DeliverPushActive() == push
        with pytest.raises(ValueError, match="calibration"):
            ngpu.SetDeliverPush(not push)
        counts = np.asarray(ngpu.GetStatus(n, "spike_count")).ravel()
        res.append((counts, np.asarray(ngpu.GetRecordData(rec), dtype=np.float32), ngpu.GetStats()))
    (c1, r1, s1), (c2, r2, s2) = res
    assert c1.sum() > 500
    assert np.array_equal(c1, c2)
    assert np.array_equal(r1, r2)
    assert s2["n_events"] > 0 and s1["status"] == s2["status"] == 0
    assert s2["n_events"] <= s1["n_events"] <= s2["n_events"] * (1.0 + 2.0 * delay / 103.0)
    o = orc.Oracle()
    n_o = iaf_two_populations(o, delay=delay)
    o.Simulate(103.0)
    assert np.array_equal(c1, np.asarray(o.GetStatus(n_o, "spike_count")).ravel())


@pytest.mark.parametrize("occ,tpi", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_per_neuron_parameters_bitexact(occ, tpi):
    """Receptor time constants drawn per neuron (parameter arrays instead of uniform kernel
    arguments): spike counts and derivative evaluations equal the oracle's."""
    from workloads import c4_network
    ngpu.SetUpdateOccupancy(occ)
    ngpu.SetUpdateTrialIter(tpi)
    n_g = c4_network(ngpu, 5, n=300, drive_w=1.5)
    o = orc.Oracle()
    n_o = c4_network(o, 5, n=300, drive_w=1.5)
    ngpu.Simulate(40.0)
    o.Simulate(40.0)
    c_g = np.asarray(ngpu.GetStatus(n_g, "spike_count")).ravel()
    c_o = np.asarray(o.GetStatus(n_o, "spike_count")).ravel()
    assert c_g.sum() > 100
    assert np.array_equal(c_g, c_o)
    assert ngpu.GetStats()["n_derivs"] == o.NDerivs()


def test_persistent_step_loop_equals_per_batch_launches():
    """Eight iaf_psc_exp populations (minimum delay one step): the persistent cooperative
    step loop and per-batch launches give the same spikes and recorded traces."""
    from workloads import microcircuit
    res = []
    for pers in (True, False):
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        ngpu.SetDeliverPush(False)
        ngpu.SetPersistent(pers)
        pops = microcircuit(ngpu, scale=0.03)
        rec = ngpu.CreateRecord("", ["V_m_rel", "I_syn_ex", "spike"], [pops[0][0], pops[2][3], pops[4][1]],
                                [0, 0, 0])
        ngpu.Simulate(60.0)
        ngpu.Simulate(45.0)
        counts = np.concatenate([np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops])
        res.append((counts, np.asarray(ngpu.GetRecordData(rec), dtype=np.float32), ngpu.GetStats()))
    (c1, r1, s1), (c2, r2, s2) = res
    assert c1.sum() > 500
    assert np.array_equal(c1, c2)
    assert np.array_equal(r1, r2)
    assert s1["n_events"] == s2["n_events"] and s1["status"] == 0


def test_persistent_barrier_timeout_is_reported():
    """Failure path of the persistent step loop: barriers told to wait for one block more
    than the launch has run out of polls; Simulate fails with an error instead of hanging,
    and the engine (and its GPU context) keeps working afterwards."""
    from workloads import microcircuit
    ngpu.SetDeliverPush(False)
    ngpu.SetPersistent(True)
    ngpu._c["NGPU_TestBarrierTimeout"](1)
    microcircuit(ngpu, scale=0.01)
    with pytest.raises(ValueError, match="timed out"):
        ngpu.Simulate(1.0)
    ngpu._c["NGPU_TestBarrierTimeout"](0)
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    ngpu.SetHostRng(True)
    pops_g = microcircuit(ngpu, scale=0.02)
    o = orc.Oracle()
    pops_o = microcircuit(o, scale=0.02)
    ngpu.Simulate(50.0)
    o.Simulate(50.0)
    c_g = np.concatenate([np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops_g])
    c_o = np.concatenate([np.asarray(o.GetStatus(p, "spike_count")).ravel() for p in pops_o])
    assert np.array_equal(c_g, c_o)


def test_mapping_change_between_calls_keeps_results():
    """Launch-mapping knobs set between Simulate calls take effect (the captured graphs are
    dropped) and change nothing in the results: 60 + 90 ms under two mappings equal the same
    two calls under the default mapping, and GetLaunchMapping reports the new mapping."""
    ref = _continuation(ngpu, [60.0, 90.0])
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)

    class Switch(object):
        """Forwards to the engine; from the second Simulate call on, under another mapping."""
        calls = 0

        def __getattr__(self, name):
            return getattr(ngpu, name)

        def Simulate(self, t):
            if self.calls:
                ngpu.SetUpdateThreads(256)
                ngpu.SetDeliverGroup(8)
                ngpu.SetUpdateOccupancy(1)
                ngpu.SetRk5Budget(2)
            self.calls += 1
            ngpu.Simulate(t)

    out = _continuation(Switch(), [60.0, 90.0])
    m = ngpu.GetLaunchMapping()
    assert m["update_threads"] == 256 and m["deliver_group"] == 8 and m["update_occupancy"] == 1
    assert m["rk5_budget"] == 2
    assert ref[0].sum() > 0
    for a, b in zip(ref, out):
        assert np.array_equal(a, b)


def _rate_change(api):
    api.SetKernelStatus("rnd_seed", 21)
    pg = api.Create("poisson_generator")
    api.SetStatus(pg, "rate", 6000.0)
    n = api.Create("aeif_cond_beta_multisynapse", 80, 2)
    api.SetStatus(n, {"E_rev": [0.0, -85.0]})
    api.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 0.6, "delay": 1.0})
    api.Connect(n, n, {"rule": "fixed_total_number", "total_num": 600}, {"weight": 0.4, "delay": 1.5})
    api.ActivateSpikeCount(n)
    counts = []
    for rate in (6000.0, 14000.0, 3000.0):
        api.SetStatus(pg, "rate", rate)
        api.Simulate(60.0)
        counts.append(np.asarray(api.GetStatus(n, "spike_count")).ravel().copy())
    return counts


def test_generator_rate_change_between_calls():
    """A poisson_generator rate set between Simulate calls applies from the next call (the
    generator table is device data: the captured graphs stay), as in the oracle."""
    c_gpu = _rate_change(ngpu)
    c_orc = _rate_change(orc.Oracle())
    for a, b in zip(c_gpu, c_orc):
        assert np.array_equal(a, b)
    assert c_gpu[1].sum() - c_gpu[0].sum() > c_gpu[0].sum()   # the higher rate shows


def test_spike_count_array_equals_status_list():
    ngpu.SetHostRng(True)
    c_list, _ = fixed_train_network(ngpu, model="aeif_cond_beta_multisynapse", t_sim=100.0, record=False)
    arr = ngpu.GetSpikeCountArray(ngpu.NodeSeq(0, c_list.size))   # the network's neurons come first
    assert arr.dtype == np.int32 and np.array_equal(arr, c_list) and arr.sum() > 0


@pytest.mark.parametrize("net", ["microcircuit", "aeif_poisson"])
def test_programmatic_launch_keeps_results(net):
    """Programmatic dependent launch of the batch kernels (default) and plain stream order
    give the same spikes, recorded traces and event counts: the microcircuit slice (one step
    per batch, delivery and update alternating) and an aeif network with Poisson drive
    (batch, straggler and delivery kernels)."""
    from workloads import microcircuit
    res = []
    for pdl in (True, False):
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        ngpu.SetProgrammaticLaunch(pdl)
        if net == "microcircuit":
            pops = microcircuit(ngpu, scale=0.03)
            rec = ngpu.CreateRecord("", ["V_m_rel", "I_syn_ex"], [pops[0][0], pops[2][3]], [0, 0])
            t = (60.0, 45.0)
        else:
            ngpu.SetKernelStatus("rnd_seed", 3)
            pg = ngpu.Create("poisson_generator")
            ngpu.SetStatus(pg, "rate", 12000.0)
            nodes = ngpu.Create("aeif_cond_beta_multisynapse", 200, 2)
            ngpu.SetStatus(nodes, {"E_rev": [0.0, -85.0]})
            ngpu.Connect(pg, nodes, {"rule": "all_to_all"}, {"weight": 0.4, "delay": 0.2, "receptor": 0})
            ngpu.Connect(nodes, nodes, {"rule": "fixed_total_number", "total_num": 1600},
                         {"weight": 0.2, "delay": 1.3, "receptor": 0})
            ngpu.ActivateSpikeCount(nodes)
            pops = [nodes]
            rec = ngpu.CreateRecord("", ["V_m", "w"], [nodes[0], nodes[7]], [0, 0])
            t = (40.0, 30.0)
        for ti in t:
            ngpu.Simulate(ti)
        counts = np.concatenate([np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops])
        res.append((counts, np.asarray(ngpu.GetRecordData(rec), dtype=np.float32), ngpu.GetStats()))
    (c1, r1, s1), (c2, r2, s2) = res
    assert c1.sum() > 100
    assert np.array_equal(c1, c2)
    assert np.array_equal(r1, r2)
    assert s1["n_events"] == s2["n_events"] and s1["status"] == 0 and s2["status"] == 0


@pytest.mark.parametrize("nport", [1, 2, 5, 8, 20])
@pytest.mark.parametrize("model", MODELS[:4])
def test_many_receptor_ports_bitexact(model, nport):
    """Receptor counts from 1 up to the reference's maximum of 20 (compile-time port counts up
    to 4, the runtime-port kernel above): spike counts and the recorded membrane potential and
    first- and last-port inputs equal the oracle's bit for bit."""
    from scenarios import many_port_network
    c_gpu, d_gpu = many_port_network(ngpu, model, nport)
    c_orc, d_orc = many_port_network(orc.Oracle(), model, nport)
    assert c_gpu.sum() > 0
    assert np.array_equal(c_gpu, c_orc)
    assert np.array_equal(np.float32(d_gpu), np.float32(d_orc))
    assert ngpu.GetStats()["status"] == 0


def _iaf_singular(api, tau_ex):
    """iaf_psc_exp neurons whose excitatory synaptic time constant equals (or nearly equals)
    the membrane time constant: the propagator's singular branch
    (src/propagator_stability.cu:31-52)."""
    n = api.Create("iaf_psc_exp", 2)
    api.SetStatus(n, {"tau_m": 10.0, "tau_ex": tau_ex, "C_m": 250.0})
    sg = api.Create("spike_generator")
    api.SetStatus(sg, {"spike_times": [1.0, 4.0, 4.5, 12.0]})
    api.Connect(sg, n, {"rule": "all_to_all"}, {"weight": 300.0, "delay": 1.0, "receptor": 0})
    rec = api.CreateRecord("", ["V_m_rel", "V_m_rel"], [n[0], n[1]], [0, 0])
    api.Simulate(40.0)
    return np.asarray(api.GetRecordData(rec), dtype=np.float64)[:, 1], n


@pytest.mark.parametrize("tau_ex", [10.0, 10.05])
def test_iaf_propagator_singular_branch(tau_ex):
    v_gpu, n = _iaf_singular(ngpu, tau_ex)
    v32, _ = _iaf_singular(orc.Oracle(fp64=False), tau_ex)
    v64, _ = _iaf_singular(orc.Oracle(fp64=True), tau_ex)
    assert np.array_equal(np.float32(v_gpu), np.float32(v32))
    assert np.max(np.abs(v_gpu - v64)) / np.max(np.abs(v64)) < 1e-5
    assert v_gpu.max() > 1.0
    if tau_ex == 10.0:
        # P21ex = h / C_m * exp(-h / tau) in the singular case
        p21 = float(np.ravel(ngpu.GetStatus(n[0], "P21ex"))[0])
        assert abs(p21 - 0.1 / 250.0 * math.exp(-0.1 / 10.0)) < 1e-9


def _aeif_guard(api):
    """aeif neurons started outside the ExternalUpdate guard bounds
    (src/aeif_cond_beta_multisynapse_kernel.h:196-207): V_m < -1e3 mV, w > 1e6 pA, w < -1e6 pA
    and one neuron inside them.  The guard resets V_m to V_reset and w to 0."""
    n = api.Create("aeif_cond_beta_multisynapse", 4, 2)
    api.SetStatus(n, {"E_rev": [0.0, -85.0], "I_e": 300.0})
    api.SetStatus(n[0:1], {"V_m": -2000.0})
    api.SetStatus(n[1:2], {"w": 2.0e6})
    api.SetStatus(n[2:3], {"w": -2.0e6})
    rec = api.CreateRecord("", ["V_m"] * 4 + ["w"] * 4, [n[i] for i in range(4)] * 2, [0] * 8)
    api.Simulate(5.0)
    return np.asarray(api.GetRecordData(rec), dtype=np.float64)


def test_aeif_state_guard_resets():
    d_gpu = _aeif_guard(ngpu)
    d_orc = _aeif_guard(orc.Oracle(fp64=False))
    assert np.array_equal(np.float32(d_gpu), np.float32(d_orc))
    assert ngpu.GetStats()["status"] & 4        # the numeric-guard status bit
    # after the first step the three guarded neurons sit near V_reset with w near 0
    row = d_gpu[1]
    for i in range(3):
        assert abs(row[1 + i] + 60.0) < 5.0 and abs(row[5 + i]) < 10.0
    assert abs(row[4] + 70.6) < 5.0


@pytest.mark.parametrize("query_first", [False, True])
def test_device_rule_expansion_keeps_connections(query_first):
    """Connect calls expanded on the device (every fixed_total_number / fixed_indegree /
    fixed_outdegree call, whatever its size) list the same connections, in the reference's
    order, as the host path: queried after calibration (the device blocks are brought to the
    host store then) or before it (the calibration then reads the host store)."""
    from ref_runner import conn_arrays, rules_network
    ngpu.SetDeviceRuleMinEdges(1 << 62)
    rules_network(4321)
    ngpu.Calibrate()
    host = conn_arrays()
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    ngpu.SetDeviceRuleMinEdges(0)
    rules_network(4321)
    if query_first:
        early = conn_arrays()
    ngpu.Calibrate()
    dev = conn_arrays()
    for k in ("source", "group", "index", "target", "port"):
        assert dev[k] == host[k], k
        if query_first:
            assert early[k] == host[k], k
    assert np.array_equal(np.float32(dev["weight"]), np.float32(host["weight"]))
    assert np.array_equal(np.float32(dev["delay"]), np.float32(host["delay"]))


def test_microcircuit_slice_device_rules_bitexact():
    """The microcircuit slice with every projection expanded on the device gives the same
    spikes as with the host expansion of the same cuRAND draws."""
    from workloads import microcircuit
    counts = []
    for min_edges in (1 << 62, 0):
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        ngpu.SetDeviceRuleMinEdges(min_edges)
        pops = microcircuit(ngpu, scale=0.03)
        ngpu.Simulate(150.0)
        counts.append(np.concatenate([np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops]))
        assert ngpu.GetStats()["status"] == 0
    assert counts[0].sum() > 1000
    assert np.array_equal(counts[0], counts[1])


def test_spike_detector_matches_oracle():
    """spike_detector nodes (src/spike_detector.cu) behind Poisson-driven aeif neurons, as in
    the reference's spike-time test: recorded spike heights, spike counts and recorded spike
    times equal the oracle's."""
    from scenarios import spike_detector_scenario
    d_g, c_g, t_g = spike_detector_scenario(ngpu)
    d_o, c_o, t_o = spike_detector_scenario(orc.Oracle())
    assert c_g.sum() > 0
    assert np.array_equal(c_g, c_o)
    assert np.array_equal(np.float32(d_g), np.float32(d_o))
    assert np.array_equal((d_g[:, 1:] > 0.5).sum(axis=0), c_g)
    for a, b in zip(t_g, t_o):
        assert np.array_equal(np.float32(a), np.float32(b))
