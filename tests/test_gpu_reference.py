"""The engine against the reference's own CUDA build on the same GPU.

oracle/_ref/libnestgpukernel.so is compiled from the reference sources by
oracle/Makefile.ref (at build time, where the sources are present) and travels
with the repository; each scenario runs in a child process through the same
nestgpu.py interface with NESTGPU_LIB pointing at it.  Skipped when that
library was not built.

Compared: the connection random stream and every connection of a rule-based
network (bit-exact), single-neuron traces (1e-5 relative), and spike counts of
recurrent networks driven by fixed spike trains (exact).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import nestgpu as ngpu
from scenarios import fixed_train_network, plastic_network, stdp_pair_scenario, trace_scenario

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnestgpukernel.so")
RUNNER = os.path.join(ROOT, "tests", "ref_runner.py")

needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")


def run_reference(what, timeout=600):
    env = dict(os.environ, NESTGPU_LIB=REF_LIB)
    p = subprocess.run([sys.executable, RUNNER, what], env=env, capture_output=True, text=True,
                       timeout=timeout)
    assert p.returncode == 0, p.stderr[-2000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("JSON:")][-1]
    return json.loads(line[5:])


def run_own(what, timeout=600):
    """The same scenario through this engine's library, in a child process."""
    env = dict(os.environ)
    env.pop("NESTGPU_LIB", None)
    p = subprocess.run([sys.executable, RUNNER, what], env=env, capture_output=True, text=True,
                       timeout=timeout)
    assert p.returncode == 0, p.stderr[-2000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("JSON:")][-1]
    return json.loads(line[5:])


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    yield
    ngpu.Reset()


@needs_ref
def test_random_stream_matches_reference():
    ref = run_reference("random:2024")
    ngpu.SetRandomSeed(2024)
    assert [int(x) for x in ngpu.RandomInt(1000)] == ref["int"]
    assert np.array_equal(np.float32(ngpu.RandomNormal(1001, 0.5, 2.0)), np.float32(ref["normal"]))


@needs_ref
def test_connectivity_matches_reference():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ref_runner import conn_arrays, rules_network
    ref = run_reference("rules")
    rules_network(4321)
    got = conn_arrays()
    for k in ("source", "group", "index", "target", "port"):
        assert got[k] == ref[k], k
    assert np.array_equal(np.float32(got["weight"]), np.float32(ref["weight"]))
    assert np.array_equal(np.float32(got["delay"]), np.float32(ref["delay"]))


@needs_ref
@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "iaf_psc_exp"])
def test_trace_close_to_reference(model):
    ref = run_reference("trace:" + model)
    _, v = trace_scenario(ngpu, model)
    vr = np.asarray(ref["v"])
    assert np.max(np.abs(v - vr) / np.maximum(np.abs(vr), 1.0)) < 1e-5


@needs_ref
@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "iaf_psc_exp"])
def test_spike_counts_match_reference(model):
    ref = run_reference("fixed_train:" + model)
    counts, _ = fixed_train_network(ngpu, model=model)
    assert counts.sum() > 0
    assert counts.tolist() == ref["counts"]


@needs_ref
def test_stdp_pairs_match_reference():
    """The reference's STDP known-answer scenario (python/test/test_stdp.py) run by the
    reference build and by this engine.  Both are within the test's 1e-5 of the closed form,
    and the weights agree bit for bit except where a post-synaptic spike sits on a step
    boundary: the tiny plastic EPSP then moves it one step in one build and not in the other
    (the FP32 arithmetic differs: CUDA's expf there, the engine's own exp here), which shows
    as the closed-form weight for Dt - 0.1 ms."""
    ref = run_reference("stdp_pairs")
    dts, w, exp = stdp_pair_scenario(ngpu)
    w_ref = np.asarray(ref["weight"])
    assert np.max(np.abs(w_ref - np.asarray(ref["expected"]))) < 1e-5
    assert np.max(np.abs(w - exp)) < 1e-5
    same = w == w_ref
    assert same.sum() >= len(w) - 2
    for i in np.nonzero(~same)[0]:
        # each build's weight is the closed form at Dt or at Dt one step (0.1 ms) off
        cands = [exp[i]] + [stdp_pair_scenario_weight(dts[i] + s) for s in (-0.1, 0.1)]
        assert all(min(abs(x - c) for c in cands) < 1e-9 for x in (w[i], w_ref[i]))


def stdp_pair_scenario_weight(dt_ms):
    from scenarios import STDP_PAR, stdp_expected
    p = STDP_PAR
    return stdp_expected(p["Wmax"] / 2, dt_ms, p["tau_plus"], p["tau_minus"], p["lambda"], p["alpha"],
                         p["mu_plus"], p["mu_minus"], p["Wmax"])


@needs_ref
@pytest.mark.parametrize("case", [1, 3, 5, 6, 8, 10])
def test_stdp_cases_match_reference(case):
    """The reference's STDP cases (parrot neurons, dendritic delays of 1 and 3 ms) run by the
    reference build and by this engine: the same weight to 1e-6."""
    from scenarios import stdp_case
    ref = run_reference("stdp_case:%d" % case)
    w = stdp_case(ngpu, case)
    assert abs(w - ref["weight"]) <= 1e-6 * abs(ref["weight"])


@needs_ref
@pytest.mark.parametrize("model", ["aeif_cond_beta_multisynapse", "iaf_psc_exp"])
def test_plastic_network_matches_reference(model):
    """A recurrent network with plastic excitatory edges under fixed input trains: spike counts
    equal the reference build's exactly.  iaf_psc_exp (exact propagators, no transcendental
    functions in the step) gives the same weights; for aeif, whose threshold crossings depend
    on the FP32 exp, at least 97% of the plastic weights are bit-identical and the others are
    edges whose pre/post spike pairs ended one step apart in the two builds."""
    ref = run_reference("plastic:" + model)
    counts, w = plastic_network(ngpu, model=model)
    w_ref = np.asarray(ref["weight"], dtype=np.float32)
    assert counts.tolist() == ref["counts"]
    if model == "iaf_psc_exp":
        assert np.allclose(w, w_ref, rtol=1e-6, atol=1e-7)
    else:
        assert np.mean(w == w_ref) >= 0.97


@needs_ref
def test_network_rate_and_isi_cv_match_reference():
    """Chaotic regime: the benchmark network at 1/10 size (100k AdEx neurons, ~20 Hz),
    1 s after a 200 ms transient.  Poisson streams differ by design (Philox vs cuRAND), so
    the comparison is statistical: mean rate and mean ISI CV of 2000 neurons within 2%."""
    ref = run_reference("stats:0.1:1000", timeout=900)
    own = run_own("stats:0.1:1000")
    assert own["rate_hz"] > 5.0 and own["n_cv"] > 500
    assert abs(own["rate_hz"] - ref["rate_hz"]) <= 0.02 * ref["rate_hz"]
    assert abs(own["isi_cv"] - ref["isi_cv"]) <= 0.02 * ref["isi_cv"]


@needs_ref
def test_microcircuit_rates_match_reference():
    """The iaf_psc_exp microcircuit at 1/10 size: mean rate over all populations within 2%
    of the reference build's, each population within 10% (a few hundred neurons each)."""
    ref = run_reference("microcircuit:0.1:1000", timeout=900)
    own = run_own("microcircuit:0.1:1000")
    r_ref, r_own = np.array(ref["pop_rates_hz"]), np.array(own["pop_rates_hz"])
    n = np.round(np.array([20683, 5834, 21915, 5479, 4850, 1065, 14395, 2948]) * 0.1)
    mean_ref, mean_own = (r_ref * n).sum() / n.sum(), (r_own * n).sum() / n.sum()
    assert abs(mean_own - mean_ref) <= 0.02 * mean_ref
    assert np.all(np.abs(r_own - r_ref) <= 0.10 * np.maximum(r_ref, 1.0))
