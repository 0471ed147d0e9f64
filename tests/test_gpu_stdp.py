"""STDP on the GPU against the reference's known-answer test and the oracle.

Plastic edges (synapse groups) are depressed when a spike arrives after the target's last
spike (src/get_spike.cu:85-95) and potentiated when the target spikes after the edge's last
arrival (src/rev_spike.cu:46-92), with the Guetig rule of src/stdp.cu:36-64 computed in
FP64.  The engine and the oracle apply the same updates in the same step order; the FP64
exp/pow come from CUDA on one side and from the C library on the other, so plastic weights
are compared within 1e-6 relative (they agree to the last float bit unless an FP64 last-place
difference crosses a float rounding boundary), spike counts exactly."""
import numpy as np
import pytest

import nestgpu as ngpu
import oracle as orc
from scenarios import STDP_PAR, plastic_network, stdp_pair_scenario

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    yield
    ngpu.Reset()


def test_stdp_pairs_match_closed_form_and_oracle():
    dts, w, exp = stdp_pair_scenario(ngpu)
    assert np.max(np.abs(w - exp)) < 1e-5            # the reference test's tolerance
    _, w_orc, _ = stdp_pair_scenario(orc.Oracle())
    assert np.allclose(w, w_orc, rtol=1e-6, atol=0.0)
    assert ngpu.GetBatchLength() == 1


def test_stdp_exponents_and_asymmetry():
    par = dict(STDP_PAR, mu_plus=0.4, mu_minus=1.7, alpha=0.6, tau_minus=35.0)
    _, w, exp = stdp_pair_scenario(ngpu, par=par)
    assert np.max(np.abs(w - exp)) < 1e-5


@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "iaf_psc_exp"])
def test_plastic_network_matches_oracle(model):
    c_gpu, w_gpu = plastic_network(ngpu, model=model)
    c_orc, w_orc = plastic_network(orc.Oracle(), model=model)
    assert c_gpu.sum() > 100
    assert np.array_equal(c_gpu, c_orc)
    assert np.allclose(w_gpu, w_orc, rtol=1e-6, atol=1e-9)
    assert np.std(w_gpu) > 0.01


def test_plastic_network_independent_of_graph_length():
    ngpu.SetGraphSteps(7)
    c7, w7 = plastic_network(ngpu, t_sim=200.0)
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    c1, w1 = plastic_network(ngpu, t_sim=200.0)
    assert np.array_equal(c7, c1)
    assert np.array_equal(w7, w1)


def _test_model_net(api):
    api.SetKernelStatus("rnd_seed", 77)
    g = api.CreateSynGroup("test_syn_model", {"fact": 0.02, "offset": -0.001})
    n = api.Create("iaf_psc_exp", 40)
    for i in range(40):
        api.SetStatus([n[i]], {"I_e": 372.0 + 0.7 * i})
    api.Connect(n, n, {"rule": "fixed_indegree", "indegree": 5},
                {"weight": 20.0, "delay": 1.0, "synapse_group": g})
    api.ActivateSpikeCount(n)
    api.Simulate(300.0)
    ids = api.GetConnections(n, n)
    st = getattr(api, "GetConnStatusList", None)
    w = st(ids, "weight") if st is not None else api.GetStatus(ids, "weight")
    return np.asarray(api.GetStatus(n, "spike_count")).ravel(), np.asarray(w, dtype=np.float32)


def test_linear_test_synapse_model_bitexact():
    c_gpu, w_gpu = _test_model_net(ngpu)
    c_orc, w_orc = _test_model_net(orc.Oracle())
    assert c_gpu.sum() > 50
    assert np.array_equal(c_gpu, c_orc)
    assert np.array_equal(w_gpu, w_orc)
    assert np.any(w_gpu != 20.0)


def test_stamp_wraparound_matches_oracle():
    """7 s of plastic edges: the stamp resets at 2^15 and 2^16 steps run on the device as in
    the oracle; edges without (recent) arrivals stay inert."""
    from scenarios import stdp_wrap_network
    w = stdp_wrap_network(ngpu)
    w_orc = stdp_wrap_network(orc.Oracle())
    assert np.allclose(w, w_orc, rtol=1e-6, atol=1e-9)
    assert np.all(w.reshape(6, 4)[4] == 1.0)


@pytest.mark.parametrize("case", list(range(1, 11)))
def test_reference_stdp_cases(case):
    """The reference's STDP cases (parrot neurons, dendritic delays): the closed form and the
    oracle."""
    from scenarios import stdp_case, stdp_case_expected
    w = stdp_case(ngpu, case)
    assert abs(w - stdp_case_expected(case)) < 1e-5
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    assert abs(w - stdp_case(orc.Oracle(), case)) <= 1e-6 * abs(w)


def test_parrot_neuron_matches_oracle():
    from scenarios import parrot_scenario
    c_gpu, r_gpu = parrot_scenario(ngpu)
    c_orc, r_orc = parrot_scenario(orc.Oracle())
    assert c_gpu.tolist() == c_orc.tolist() and c_gpu[1] == 0 and c_gpu[0] > 0
    assert np.array_equal(np.float32(r_gpu), np.float32(r_orc))


def test_plastic_network_with_dendritic_delays_matches_oracle():
    from scenarios import plastic_den_delay_network
    c_gpu, w_gpu = plastic_den_delay_network(ngpu)
    c_orc, w_orc = plastic_den_delay_network(orc.Oracle())
    assert c_gpu.sum() > 100
    assert np.array_equal(c_gpu, c_orc)
    assert np.allclose(w_gpu, w_orc, rtol=1e-6, atol=1e-9)


def test_linear_test_synapse_like_reference():
    """python/test/test_syn_model.py on the GPU: w = dt * fact + offset within its 1e-6."""
    from scenarios import syn_model_scenario
    w, exp = syn_model_scenario(ngpu)
    assert np.max(np.abs(w - exp)) < 1e-6
