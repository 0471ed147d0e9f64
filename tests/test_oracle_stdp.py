"""The oracle's synapse groups and STDP pinned against the reference's known-answer test
(python/test/test_stdp.py: one pre/post pair per time difference, weights against the
closed-form Guetig rule within the reference's 1e-5).  CPU only."""
import numpy as np
import pytest

import oracle as orc
from scenarios import STDP_PAR, plastic_network, stdp_pair_scenario


@pytest.mark.parametrize("fp64", [False, True])
def test_stdp_pairs_match_closed_form(fp64):
    dts, w, exp = stdp_pair_scenario(orc.Oracle(fp64=fp64))
    assert np.max(np.abs(w - exp)) < 1e-5
    # both branches are exercised and the weights moved
    assert np.sum(np.asarray(dts) < 0) > 10 and np.sum(np.asarray(dts) > 0) > 10
    w0 = STDP_PAR["Wmax"] / 2
    assert np.all(w[np.asarray(dts) < 0] < w0) and np.all(w[np.asarray(dts) > 0] > w0)


def test_stdp_weight_dependence_exponents():
    par = dict(STDP_PAR, mu_plus=0.4, mu_minus=1.7, alpha=0.6, tau_minus=35.0)
    _, w, exp = stdp_pair_scenario(orc.Oracle(), par=par)
    assert np.max(np.abs(w - exp)) < 1e-5


def test_synapse_group_parameters():
    o = orc.Oracle()
    g = o.CreateSynGroup("stdp")
    assert abs(o.GetStatus(g, "Wmax") - 100.0) < 1e-6 and abs(o.GetStatus(g, "lambda") - 1e-4) < 1e-10
    o.SetStatus(g, {"Wmax": 3.0})
    assert o.GetStatus(g, "Wmax") == 3.0
    with pytest.raises(ValueError):
        o.CreateSynGroup("no_such_model")
    with pytest.raises(ValueError):
        o.GetStatus(g, "no_such_param")


@pytest.mark.parametrize("model,wmax", [("aeif_cond_beta_multisynapse", 3.0), ("iaf_psc_exp", 80.0)])
def test_plastic_network_moves_weights(model, wmax):
    counts, w = plastic_network(orc.Oracle(), model=model)
    assert 5.0 < counts.sum() / counts.size / 0.4 < 200.0
    assert np.std(w) > 0.05 * wmax / 3 and np.all(w >= 0.0) and np.all(w <= wmax)


def test_stamp_resets_keep_old_and_missing_arrivals_inert():
    """After 2^15 and 2^16 steps the 16-bit stamps are reset (src/nestgpu.cu:490-498): an edge
    that never carried a spike and an edge whose last spike is older than 2^16 steps see no
    potentiation from the later postsynaptic spikes."""
    from scenarios import stdp_wrap_network
    w = stdp_wrap_network(orc.Oracle()).reshape(6, 4)
    w_early = stdp_wrap_network(orc.Oracle(), t_sim=400.0).reshape(6, 4)
    assert np.all(w[4] == 1.0)
    assert np.array_equal(w[5], w_early[5]) and np.any(w_early[5] != 1.0)
    assert np.std(w[0:4]) > 0.01


@pytest.mark.parametrize("case", list(range(1, 11)))
def test_reference_stdp_cases(case):
    """python/test/test_stdp/cases/case<N>.py: parrot neurons, dendritic delays of 1 and 3 ms,
    depression and potentiation sequences; the weight against the cases' closed form."""
    from scenarios import stdp_case, stdp_case_expected
    assert abs(stdp_case(orc.Oracle(), case) - stdp_case_expected(case)) < 1e-5


def test_parrot_neuron_repeats_port0_only():
    """src/parrot_neuron.cu:60-82: a spike arriving on port 0 is repeated one step after the
    step it arrives in (height 1 unless hold_spike_height); port 1 input is weighted 0."""
    o = orc.Oracle()
    sg = o.Create("spike_generator")
    p = o.Create("parrot_neuron", 3)
    o.SetStatus(sg, {"spike_times": [2.0, 5.0], "spike_heights": [2.0, 3.0]})
    o.Connect(sg, p[0:1], {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    o.Connect(sg, p[1:2], {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0, "receptor": 1})
    o.Connect(sg, p[2:3], {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    o.SetStatus(p[2:3], {"hold_spike_height": 1.0})
    o.ActivateSpikeCount(p)
    rec = o.CreateRecord("", ["V", "V", "V"], [p[0], p[1], p[2]], [0, 0, 0])
    o.Simulate(10.0)
    assert o.GetStatus(p, "spike_count") == [2, 0, 2]
    v = np.asarray(o.GetRecordData(rec))
    # the V column holds the repeated input in the step where the parrot fires
    assert sorted(set(np.round(v[:, 1], 3))) == [0.0, 2.0, 3.0]
    assert np.all(v[:, 2] == 0.0)


def test_linear_test_synapse_like_reference():
    """python/test/test_syn_model.py: w = dt * fact + offset within its 1e-6."""
    from scenarios import syn_model_scenario
    w, exp = syn_model_scenario(orc.Oracle())
    assert np.max(np.abs(w - exp)) < 1e-6
