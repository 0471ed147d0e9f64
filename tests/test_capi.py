"""C ABI and host-side logic of the engine (runs without a GPU).

Connection rules, the connection store's reference ordering, parameter and
variable bookkeeping and error behaviour are host code; they are checked here
against the oracle and the reference's golden connect log.  No kernel runs.
"""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import nestgpu as ngpu
import oracle as orc
from scenarios import GOLDEN, connect_scenario

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nestgpu_b200.h")


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    yield
    ngpu.Reset()


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:NESTGPU|NGPU)_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(ngpu.lib_path)
    syms = declared_symbols()
    assert len([s for s in syms if s.startswith("NESTGPU_")]) == 133
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_connect_log_golden_through_engine():
    gold = json.load(open(os.path.join(GOLDEN, "connect_log.json")))
    got = connect_scenario(ngpu)
    assert list(gold) == list(got)
    for sec in gold:
        assert len(gold[sec]) == len(got[sec])
        for a, b in zip(gold[sec], got[sec]):
            if isinstance(a, dict):
                assert {k: a[k] for k in ("source", "target", "port", "syn")} == \
                       {k: b[k] for k in ("source", "target", "port", "syn")}
                assert a["delay"] == pytest.approx(b["delay"], rel=1e-6)
                assert a["weight"] == pytest.approx(b["weight"], rel=1e-6)
            else:
                assert a == pytest.approx(b, rel=1e-6)


def _build_rules(api, seed):
    api.SetKernelStatus("rnd_seed", seed)
    a = api.Create("aeif_cond_beta_multisynapse", 40, 2)
    b = api.Create("iaf_psc_exp", 25)
    api.Connect(a, b, {"rule": "fixed_indegree", "indegree": 7}, {"weight": 1.5, "delay": 1.0})
    api.Connect(a, a, {"rule": "fixed_indegree", "indegree": 30}, {"weight": 0.25, "delay": 0.7,
                                                                  "receptor": 1})
    api.Connect(b, a, {"rule": "fixed_outdegree", "outdegree": 5}, {"weight": 2.0, "delay": 2.0})
    api.Connect(b, b, {"rule": "fixed_total_number", "total_num": 60},
                {"weight": -1.0, "delay": {"distribution": "normal_clipped", "mu": 1.5, "sigma": 0.5,
                                           "low": 0.3, "high": 3.0, "step": 0.1}})
    api.Connect([a[3], a[5], a[9]], [b[0], b[2]], {"rule": "all_to_all"},
                {"weight": {"array": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]}, "delay": 0.5})
    api.Connect(a[0:10], b[0:10], {"rule": "one_to_one"}, {"weight": 0.5, "delay": 3.0})


def test_connection_rules_match_oracle():
    """fixed_indegree (both sampling methods), fixed_outdegree, fixed_total_number,
    all_to_all with weight arrays, one_to_one, normal_clipped delays: the engine's
    connection store equals the oracle's, in reference order."""
    ngpu.SetHostRng(True)
    _build_rules(ngpu, 1234)
    o = orc.Oracle()
    _build_rules(o, 1234)
    ref = o.ConnectionArrays()
    ids = ngpu.GetConnections()
    assert len(ids) == ref["source"].size
    st = [ngpu.GetConnectionStatus(c) for c in ids]
    assert [c.i_source for c in ids] == list(ref["source"])
    assert [c.i_group for c in ids] == list(ref["group"])
    assert [c.i_conn for c in ids] == list(ref["index"])
    assert [s["target"] for s in st] == list(ref["target"])
    assert [s["port"] for s in st] == list(ref["port"])
    assert np.array_equal(np.array([s["weight"] for s in st], dtype=np.float32), ref["weight"])
    assert np.array_equal(np.array([s["delay"] for s in st], dtype=np.float32), ref["delay"])


def test_fixed_indegree_same_sources_for_all_targets():
    src = ngpu.Create("iaf_psc_exp", 1000)
    tgt = ngpu.Create("iaf_psc_exp", 10)
    ngpu.Connect(src, tgt, {"rule": "fixed_indegree", "indegree": 50}, {"weight": 1.0, "delay": 1.0})
    per = {}
    for c in ngpu.GetConnections(src, tgt):
        per.setdefault(ngpu.GetStatus(c, "target"), set()).add(c.i_source)
    sets = list(per.values())
    assert len(sets) == 10 and all(s == sets[0] for s in sets) and len(sets[0]) == 50


def test_random_int_stream_matches_oracle():
    ngpu.SetHostRng(True)
    ngpu.SetRandomSeed(99)
    o = orc.Oracle()
    o.SetRandomSeed(99)
    assert list(o.RandomInt(257)) == ngpu.RandomInt(257)
    assert np.array_equal(o.RandomNormal(11, 1.0, 2.0), np.array(ngpu.RandomNormal(11, 1.0, 2.0),
                                                                   dtype=np.float32))


def test_parameters_and_names_before_calibration():
    n = ngpu.Create("aeif_cond_beta_multisynapse", 4, 3)
    assert ngpu.GetScalVarNames(n[0]) == ["V_m", "w"]
    assert ngpu.GetPortVarNames(n[0]) == ["g", "g1"]
    assert ngpu.GetPortParamNames(n[0]) == ["E_rev", "tau_rise", "tau_decay", "g0"]
    assert ngpu.GetGroupParamNames(n[0]) == ["h_min_rel", "h0_rel"]
    assert "refractory_step" in ngpu.GetScalParamNames(n[0])
    ngpu.SetStatus(n, {"V_th": -52.0, "E_rev": [0.0, -85.0, 10.0], "I_e": 5.0})
    ngpu.SetStatus([n[1], n[3]], "C_m", 300.0)
    assert ngpu.GetStatus(n, "V_th") == [pytest.approx(-52.0)] * 4
    assert ngpu.GetStatus(n, "C_m") == [281.0, 300.0, 281.0, 300.0]
    assert ngpu.GetStatus(n[2], "E_rev") == [0.0, -85.0, 10.0]
    assert ngpu.GetStatus(n, "V_m") == [pytest.approx(-70.6)] * 4
    assert ngpu.GetNeuronGroupParam(n[0], "h_min_rel") == pytest.approx(1e-3)
    ngpu.SetStatus(n, {"h0_rel": 0.05})
    assert ngpu.GetStatus(n[0], "h0_rel") == pytest.approx(0.05)
    i = ngpu.Create("iaf_psc_exp", 2)
    assert ngpu.GetStatus(i, "Theta_rel") == [15.0, 15.0]
    d = ngpu.GetStatus(i[0])
    assert d["tau_m"] == 10.0 and d["t_ref"] == 2.0 and "V_m_rel" in d
    pg = ngpu.Create("poisson_generator", 2)
    ngpu.SetStatus(pg, "rate", 12.5)
    assert ngpu.GetStatus(pg, "rate") == [12.5, 12.5]
    sg = ngpu.Create("spike_generator")
    ngpu.SetStatus(sg, {"spike_times": [1.0, 2.5]})
    assert ngpu.GetStatus(sg, "spike_times") == [[1.0, 2.5]]


def test_kernel_parameters():
    assert ngpu.GetKernelStatus("time_resolution") == pytest.approx(0.1)
    ngpu.SetKernelStatus({"rnd_seed": 77, "max_spike_buffer_size": 30})
    assert ngpu.GetKernelStatus("rnd_seed") == 77
    assert ngpu.GetMaxSpikeBufferSize() == 30
    assert set(ngpu.GetFloatParamNames()) == {"time_resolution", "max_spike_num_fact",
                                              "max_spike_per_host_fact"}
    assert set(ngpu.GetIntParamNames()) == {"rnd_seed", "verbosity_level", "max_spike_buffer_size",
                                            "remote_spike_height_flag"}
    assert ngpu.GetBoolParamNames() == ["print_time"]


def test_errors_like_reference():
    a = ngpu.Create("iaf_psc_exp", 3)
    with pytest.raises(ValueError, match="Delay must be >= time resolution"):
        ngpu.Connect(a, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 0.05})
    with pytest.raises(ValueError, match="Indegree larger than number of source nodes"):
        ngpu.Connect(a, a, {"rule": "fixed_indegree", "indegree": 4}, {"weight": 1.0, "delay": 1.0})
    with pytest.raises(ValueError, match="one-to-one"):
        ngpu.Connect(a, a[0:2], {"rule": "one_to_one"}, {"weight": 1.0, "delay": 1.0})
    with pytest.raises(ValueError, match="Unknown neuron model"):
        ngpu.Create("no_such_model", 2)
    with pytest.raises(ValueError, match="Number of nodes must be greater than zero"):
        ngpu.Create("iaf_psc_exp", 0)
    with pytest.raises(ValueError):
        ngpu.SetStatus(a, "no_such_param", 1.0)
    with pytest.raises(ValueError, match="Unrecognized synapse group"):
        ngpu.Connect(a, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0, "synapse_group": 1})
    with pytest.raises(ValueError, match="Unknown synapse model"):
        ngpu.CreateSynGroup("no_such_model")
    with pytest.raises(ValueError, match="MPI"):
        ngpu.RemoteConnect(0, a, 1, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    assert ngpu.MpiId() == 0 and ngpu.MpiNp() == 1


def test_calibrate_without_gpu_fails_loudly():
    """The engine never falls back to the host: without a CUDA device calibration is an error."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    a = ngpu.Create("iaf_psc_exp", 2)
    ngpu.Connect(a, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.0})
    with pytest.raises(ValueError, match="no CUDA device"):
        ngpu.Simulate(1.0)


def test_synapse_groups_and_plastic_connections():
    """Synapse groups through the C ABI (src/nestgpu_C.h:275-287) and plastic connections in
    the connection store: defaults, parameter access, the group of each connection and the
    syn_group filter of GetConnections."""
    ngpu.Reset()
    g = ngpu.CreateSynGroup("stdp", {"Wmax": 2.0, "lambda": 0.01})
    assert ngpu.GetSynGroupNParam(g) == 7
    assert ngpu.GetSynGroupParamNames(g) == ["tau_plus", "tau_minus", "lambda", "alpha", "mu_plus",
                                              "mu_minus", "Wmax"]
    st = ngpu.GetStatus(g)
    assert st["Wmax"] == 2.0 and abs(st["lambda"] - 0.01) < 1e-9 and st["tau_plus"] == 20.0
    assert ngpu.GetSynGroupParamIdx(g, "alpha") == 3 and not ngpu.IsSynGroupParam(g, "foo")
    t = ngpu.CreateSynGroup("test_syn_model")
    assert abs(ngpu.GetStatus(t, "fact") - 0.1) < 1e-7 and ngpu.GetStatus(t, "offset") == 0.0
    a = ngpu.Create("aeif_cond_beta_multisynapse", 3, 2)
    ngpu.Connect(a, a, {"rule": "one_to_one"}, {"weight": 0.5, "delay": 1.0})
    ngpu.Connect(a, a, {"rule": "all_to_all"}, {"weight": 1.0, "delay": 1.5, "synapse_group": g})
    c = ngpu.GetConnections(a, a)
    assert len(c) == 12
    assert len(ngpu.GetConnections(a, a, syn_group=0)) == 3
    plastic = ngpu.GetConnections(a, a, syn_group=g.i_syn_group)
    assert len(plastic) == 9
    assert all(ngpu.GetStatus(x)["syn"] == g.i_syn_group for x in plastic)
    ngpu.Reset()


def test_syn_group_status_like_reference_log():
    """python/test/test_syn_group.py against its log python/test/logp3_syn_group.txt: synapse
    group parameters through CreateSynGroup / SetStatus / GetStatus / GetSynGroupParam."""
    ngpu.Reset()
    g = ngpu.CreateSynGroup("test_syn_model", {"fact": 1.0, "offset": 2.0})
    assert ngpu.GetStatus(g) == {"fact": 1.0, "offset": 2.0}
    ngpu.SetStatus(g, "fact", 3.0)
    ngpu.SetStatus(g, "offset", 4.0)
    assert ngpu.GetStatus(g) == {"fact": 3.0, "offset": 4.0}
    ngpu.SetStatus(g, {"fact": 5.0, "offset": 6.0})
    assert ngpu.GetStatus(g) == {"fact": 5.0, "offset": 6.0}
    assert ngpu.GetSynGroupParam(g, "fact") == 5.0 and ngpu.GetSynGroupParam(g, "offset") == 6.0
    assert ngpu.GetStatus(g, "fact") == 5.0 and ngpu.GetStatus(g, "offset") == 6.0
    assert ngpu.GetStatus(g, ["fact", "offset"]) == [5.0, 6.0]
    assert ngpu.GetStatus(g, ["offset", "fact"]) == [6.0, 5.0]
    ngpu.Reset()
