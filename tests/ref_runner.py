"""Run a scenario through the nestgpu Python interface and print its results as JSON.

Used by the GPU tests to drive the reference library (oracle/_ref/libnestgpukernel.so,
compiled from the reference sources by oracle/Makefile.ref) in a separate process:
the reference keeps one network per process.  The library is chosen with the
NESTGPU_LIB environment variable, so the same scenario code runs against both
libraries.

    NESTGPU_LIB=oracle/_ref/libnestgpukernel.so python tests/ref_runner.py fixed_train:iaf_psc_exp
"""
import ctypes
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "nest-gpu_b200"))

import numpy as np  # noqa: E402

import nestgpu as ngpu  # noqa: E402
from scenarios import fixed_train_network, plastic_network, stdp_pair_scenario, trace_scenario  # noqa: E402


def conn_arrays():
    ids = ngpu.GetConnections()
    st = [ngpu.GetConnectionStatus(c) for c in ids]
    return {"source": [c.i_source for c in ids], "group": [c.i_group for c in ids],
            "index": [c.i_conn for c in ids], "target": [s["target"] for s in st],
            "port": [s["port"] for s in st], "weight": [s["weight"] for s in st],
            "delay": [s["delay"] for s in st]}


def rules_network(seed):
    ngpu.SetKernelStatus("rnd_seed", seed)
    a = ngpu.Create("aeif_cond_beta_multisynapse", 40, 2)
    b = ngpu.Create("iaf_psc_exp", 25)
    ngpu.Connect(a, b, {"rule": "fixed_indegree", "indegree": 7}, {"weight": 1.5, "delay": 1.0})
    ngpu.Connect(a, a, {"rule": "fixed_indegree", "indegree": 30}, {"weight": 0.25, "delay": 0.7,
                                                                   "receptor": 1})
    ngpu.Connect(b, a, {"rule": "fixed_outdegree", "outdegree": 5}, {"weight": 2.0, "delay": 2.0})
    ngpu.Connect(b, b, {"rule": "fixed_total_number", "total_num": 60},
                 {"weight": -1.0, "delay": {"distribution": "normal_clipped", "mu": 1.5, "sigma": 0.5,
                                            "low": 0.3, "high": 3.0}})
    ngpu.Connect(a[0:10], b[0:10], {"rule": "one_to_one"}, {"weight": 0.5, "delay": 3.0})


def big_network(scale, seed):
    """1M-neuron benchmark network scaled by `scale`, through the reference C API:
    per-target random sources (numpy), uniform delays 1.0-2.0 ms, one Poisson generator."""
    n = int(1_000_000 * scale)
    ne = int(0.8 * n)
    k_exc, k_inh = 800, 200
    ngpu.SetKernelStatus("rnd_seed", seed)
    neuron = ngpu.Create("aeif_cond_beta_multisynapse", n, 2)
    ngpu.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", 8000.0)
    ngpu.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": 0.1, "delay": 1.0, "receptor": 0})
    rng = np.random.RandomState(seed)
    lib = ngpu._lib
    chunk = 20000
    for t0 in range(0, n, chunk):
        t1 = min(n, t0 + chunk)
        nt = t1 - t0
        for (lo, hi, k, w, port) in ((0, ne, k_exc, 0.05, 0), (ne, n, k_inh, 0.35, 1)):
            src = rng.randint(lo, hi, size=nt * k).astype(np.int32) + neuron.i0
            tgt = (np.repeat(np.arange(t0, t1, dtype=np.int32), k) + neuron.i0).astype(np.int32)
            dl = (rng.randint(10, 21, size=nt * k) * 0.1).astype(np.float32)
            ngpu.ConnSpecInit()
            ngpu.SetConnSpecParam("rule", 0)   # one_to_one over the edge list
            ngpu.SynSpecInit()
            ngpu.SetSynSpecIntParam("receptor", port)
            ngpu.SetSynSpecFloatParam("weight", w)
            ngpu.SetSynSpecFloatPtParam("delay_array", dl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
            lib.NESTGPU_ConnectGroupGroup(ctypes.c_void_p(src.ctypes.data), ctypes.c_int(src.size),
                                          ctypes.c_void_p(tgt.ctypes.data), ctypes.c_int(tgt.size))
            ngpu._check()
    ngpu.ActivateSpikeCount(neuron)
    return neuron


def main():
    what = sys.argv[1]
    ngpu.SetVerbosityLevel(0)
    out = {}
    if what.startswith("stdp_case:"):
        from scenarios import stdp_case
        out = {"weight": stdp_case(ngpu, int(what.split(":")[1]))}
    elif what == "stdp_pairs":
        dts, w, exp = stdp_pair_scenario(ngpu)
        out = {"dt": list(dts), "weight": [float(x) for x in w], "expected": [float(x) for x in exp]}
    elif what.startswith("plastic:"):
        counts, w = plastic_network(ngpu, model=what.split(":")[1])
        out = {"counts": counts.tolist(), "weight": [float(x) for x in w]}
    elif what.startswith("fixed_train:"):
        counts, data = fixed_train_network(ngpu, model=what.split(":", 1)[1])
        out = {"counts": counts.tolist(), "record": np.asarray(data).tolist()}
    elif what.startswith("trace:"):
        t, v = trace_scenario(ngpu, what.split(":", 1)[1])
        out = {"t": list(map(float, t)), "v": list(map(float, v))}
    elif what == "rules":
        rules_network(4321)
        out = conn_arrays()
    elif what.startswith("random:"):
        ngpu.SetRandomSeed(int(what.split(":")[1]))
        out = {"int": [int(x) for x in ngpu.RandomInt(1000)],
               "normal": [float(x) for x in ngpu.RandomNormal(1001, 0.5, 2.0)]}
    elif what.startswith("timing:"):
        _, scale, bio_ms = what.split(":")
        scale, bio_ms = float(scale), float(bio_ms)
        t0 = time.time()
        neuron = big_network(scale, 20240)
        ngpu.Calibrate()
        build = time.time() - t0
        ngpu.Simulate(10.0)   # first call: the reference's "Simulation time" starts after it
        t1 = time.time()
        ngpu.Simulate(bio_ms)
        sim = time.time() - t1
        counts = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
        out = {"build_s": build, "sim_s": sim, "bio_ms": bio_ms, "rtf": sim / (bio_ms / 1000.0),
               "n_neurons": int(counts.size), "spikes": int(counts.sum())}
    elif what.startswith("stats:"):
        # the benchmark network at `scale`: rate and ISI CV of 2000 recorded neurons
        _, scale, bio_ms = what.split(":")
        scale, bio_ms = float(scale), float(bio_ms)
        neuron = big_network(scale, 20240)
        n_rec = min(2000, len(neuron))
        # the reference records spike times only for whole groups
        ngpu.ActivateRecSpikeTimes(neuron, int(200 * (bio_ms + 200.0) / 1000.0) + 20)
        ngpu.Simulate(200.0)   # transient
        c0 = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
        ngpu.Simulate(bio_ms)
        c1 = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
        cvs = []
        for t in ngpu.GetRecSpikeTimes(neuron)[:n_rec]:
            t = np.asarray(t, dtype=np.float64)
            t = t[t > 200.0]
            if t.size >= 4:
                isi = np.diff(t)
                cvs.append(isi.std() / isi.mean())
        out = {"rate_hz": float((c1 - c0).sum()) / len(neuron) / (bio_ms / 1000.0),
               "isi_cv": float(np.mean(cvs)), "n_cv": len(cvs)}
    elif what.startswith("microcircuit:"):
        # the iaf_psc_exp microcircuit: build, a 100 ms first call, then `bio_ms` timed
        from workloads import microcircuit
        _, scale, bio_ms = what.split(":")
        scale, bio_ms = float(scale), float(bio_ms)
        t0 = time.time()
        pops = microcircuit(ngpu, scale=scale)
        ngpu.Calibrate()
        build = time.time() - t0
        if getattr(ngpu, "is_b200_engine", False) and os.environ.get("NGPU_AUTOTUNE"):
            out["mapping"] = ngpu.Autotune(500)
        ngpu.Simulate(100.0)
        c0 = [np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops]
        t1 = time.time()
        ngpu.Simulate(bio_ms)
        sim = time.time() - t1
        c1 = [np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops]
        rates = [float((b - a).sum()) / len(b) / (bio_ms / 1000.0) for a, b in zip(c0, c1)]
        out.update({"build_s": build, "sim_s": sim, "bio_ms": bio_ms, "rtf": sim / (bio_ms / 1000.0),
                    "n_neurons": int(sum(len(p) for p in pops)), "pop_rates_hz": rates})
        if getattr(ngpu, "is_b200_engine", False):
            out["device_ms_per_step"] = ngpu.GetSimDeviceMs() / (bio_ms / 0.1)
            out["profile_ms_per_step"] = ngpu.ProfileSteps(1000)
    print("JSON:" + json.dumps(out))


if __name__ == "__main__":
    main()
