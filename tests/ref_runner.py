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


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon et al., SC'11) on numpy arrays of 32-bit values held in uint64."""
    m32 = np.uint64(0xFFFFFFFF)
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) for x in (c0, c1, c2, c3))
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        c0, c1, c2, c3 = (p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & m32, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & m32
        k0 = (k0 + np.uint64(0x9E3779B9)) & m32
        k1 = (k1 + np.uint64(0xBB67AE85)) & m32
    return c0, c1, c2, c3


def generated_edges(t_lo, t_hi, k, n_src, n_steps, seed):
    """Edges of targets t_lo .. t_hi-1 of a generated per-target fixed in-degree block
    (the engine's ConnectFixedIndegreeGPU): edge kk of target t draws Philox4x32-10 keyed
    by the seed with counter (t, kk, 0, 0x9E3779B9); source offset floor(x * n_src / 2^32),
    delay step offset floor(y * n_steps / 2^32).  Returns (target, source, step) offsets."""
    t = np.repeat(np.arange(t_lo, t_hi, dtype=np.uint64), k)
    kk = np.tile(np.arange(k, dtype=np.uint64), t_hi - t_lo)
    x, y, _, _ = philox4x32_10(t, kk, np.uint64(0), np.uint64(0x9E3779B9), seed & 0xFFFFFFFF, seed >> 32)
    src = (x * np.uint64(n_src)) >> np.uint64(32)
    step = (y * np.uint64(n_steps)) >> np.uint64(32)
    return t.astype(np.int64), src.astype(np.int64), step.astype(np.int64)


def generated_network(scale, seed):
    """The benchmark network of workloads.benchmark_network with its generated blocks
    pushed through the reference C API as edge lists (one_to_one over per-edge arrays),
    so that a library without ConnectFixedIndegreeGPU simulates the identical network."""
    from workloads import (BENCH_DELAY_MAX, BENCH_DELAY_MIN, BENCH_K_EXC, BENCH_K_INH, BENCH_N_EXC,
                           BENCH_N_INH, BENCH_PG_RATE, BENCH_W_EXC, BENCH_W_INH, BENCH_W_PG)
    n_exc, n_inh = int(BENCH_N_EXC * scale), int(BENCH_N_INH * scale)
    n = n_exc + n_inh
    ngpu.SetKernelStatus("rnd_seed", seed)
    neuron = ngpu.Create("aeif_cond_beta_multisynapse", n, 2)
    ngpu.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
    pg = ngpu.Create("poisson_generator")
    ngpu.SetStatus(pg, "rate", BENCH_PG_RATE)
    ngpu.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": BENCH_W_PG, "delay": 1.0, "receptor": 0})
    dt = 0.1
    dlo = int(round(BENCH_DELAY_MIN / dt)) - 1
    n_steps = int(round(BENCH_DELAY_MAX / dt)) - 1 - dlo + 1
    lib = ngpu._lib
    chunk = 20000
    blocks = ((0, n_exc, BENCH_K_EXC, BENCH_W_EXC, 0, seed), (n_exc, n_inh, BENCH_K_INH, BENCH_W_INH, 1, seed + 7919))
    for (s0, ns, k, w, port, bseed) in blocks:
        for t0 in range(0, n, chunk):
            t1 = min(n, t0 + chunk)
            tg, sr, st = generated_edges(t0, t1, k, ns, n_steps, bseed)
            src = (sr + s0 + neuron.i0).astype(np.int32)
            tgt = (tg + neuron.i0).astype(np.int32)
            dl = ((st + dlo + 1) * np.float32(dt)).astype(np.float32)
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
    elif what.startswith("balanced_trains:"):
        # the plain small balanced network (seed 42) driven by fixed input trains
        from workloads import balanced_network
        t_sim = float(what.split(":")[1])
        neuron = balanced_network(ngpu, seed=42, drive="trains", t_sim=t_sim)
        ngpu.Simulate(t_sim)
        out = {"counts": np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel().tolist()}
    elif what.startswith("timing_gen:"):
        # the benchmark network (generated edges as lists): build, `warm` ms first call, then
        # `bio_ms` timed as the reference's "Simulation time" (wall time of Simulate)
        _, scale, warm, bio_ms = what.split(":")
        scale, warm, bio_ms = float(scale), float(warm), float(bio_ms)
        t0 = time.time()
        neuron = generated_network(scale, 20240)
        ngpu.Calibrate()
        build = time.time() - t0
        ngpu.Simulate(warm)
        c0 = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
        t1 = time.time()
        ngpu.Simulate(bio_ms)
        sim = time.time() - t1
        c1 = np.asarray(ngpu.GetStatus(neuron, "spike_count")).ravel()
        spikes = int((c1 - c0).sum())
        out = {"build_s": build, "sim_s": sim, "warm_ms": warm, "bio_ms": bio_ms, "rtf": sim / (bio_ms / 1000.0),
               "n_neurons": int(c1.size), "spikes": spikes,
               "rate_hz": spikes / c1.size / (bio_ms / 1000.0),
               "events_per_s": spikes * 1000.0 / sim}
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
        # the iaf_psc_exp microcircuit: build, a first call of `warm` ms (default 500), then `bio_ms` timed
        from workloads import microcircuit
        parts = what.split(":")
        scale, bio_ms = float(parts[1]), float(parts[2])
        warm = float(parts[3]) if len(parts) > 3 else 500.0
        t0 = time.time()
        pops = microcircuit(ngpu, scale=scale)
        ngpu.Calibrate()
        build = time.time() - t0
        if getattr(ngpu, "is_b200_engine", False) and os.environ.get("NGPU_AUTOTUNE"):
            out["mapping"] = ngpu.Autotune(500)
        ngpu.Simulate(warm)
        c0 = [np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops]
        t1 = time.time()
        ngpu.Simulate(bio_ms)
        sim = time.time() - t1
        c1 = [np.asarray(ngpu.GetStatus(p, "spike_count")).ravel() for p in pops]
        rates = [float((b - a).sum()) / len(b) / (bio_ms / 1000.0) for a, b in zip(c0, c1)]
        out.update({"build_s": build, "sim_s": sim, "warm_ms": warm, "bio_ms": bio_ms, "rtf": sim / (bio_ms / 1000.0),
                    "n_neurons": int(sum(len(p) for p in pops)), "pop_rates_hz": rates,
                    "rate_hz": float(sum(float((b - a).sum()) for a, b in zip(c0, c1))) /
                    sum(len(p) for p in pops) / (bio_ms / 1000.0)})
        if getattr(ngpu, "is_b200_engine", False):
            out["device_ms_per_step"] = ngpu.GetSimDeviceMs() / (bio_ms / 0.1)
            out["profile_ms_per_step"] = ngpu.ProfileSteps(1000)
    print("JSON:" + json.dumps(out))


if __name__ == "__main__":
    main()
