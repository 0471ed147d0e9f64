"""Benchmark: 1,000,000 aeif_cond_beta_multisynapse neurons x 1000 synapses on one B200.

Workload (1 GPU): 800k excitatory + 200k inhibitory AdEx neurons with two beta
receptors (E_rev 0 / -85 mV, reference default parameters), every neuron with
800 excitatory inputs (0.05 nS, receptor 0) and 200 inhibitory inputs (0.35 nS,
receptor 1), sources drawn per target, delays uniform on {1.0, 1.1, ..., 2.0} ms
(1e9 synapses, fp32 weights), one poisson_generator at 8 kHz into every neuron
(0.1 nS, receptor 0), dt = 0.1 ms, seeded synthetic network.

A bench "step" is 100 ms of biological time (1000 integration steps of dt)
simulated through the engine's Simulate call.  `value` is synaptic events per
second (device time, whole job: replicas on every GPU add up); RTF and RK5
derivative evaluations per neuron-ms are reported next to it.  The network's
CSR (8 GB) is far larger than L2, so no flush is needed between steps.

`--impl reference` times the CPU implementation of the same path (the oracle
restatement of the reference algorithm, OpenMP over the host cores) on a
bounded sample of the workload: 20,000 neurons with the same in-degree, rates
and delays for 100 ms of biological time per step; events/s and the RTF
extrapolated per neuron are reported.

Multi-GPU (torchrun): by default each rank simulates its own replica (different
seed); no collective is on the data path, only a barrier and a max-reduction of the
step time (weak scaling).  With --partition the ranks simulate one network together:
each rank its share of the neurons with their in-edges, the spikes of every time batch
all-gathered over NCCL (nest-gpu_b200/partition.py; strong scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
RANK = int(os.environ.get("RANK", "0"))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))

N_EXC, N_INH = 800_000, 200_000
K_EXC, K_INH = 800, 200
W_EXC, W_INH, W_PG = 0.05, 0.35, 0.1
PG_RATE = 8000.0
DELAY_MIN, DELAY_MAX = 1.0, 2.0
STEP_MS = 100.0
FLOPS_PER_DERIV = 110        # FP32 flops per derivative evaluation incl. stage algebra, 2 ports
DELIVERY_BYTES_PER_EVENT = 8  # 4 B packed target/port + 4 B weight per synaptic event
DELIVERY_BYTES_PER_SPIKE = 8  # ring entry (source, height)
# DRAM traffic per unit (dram__bytes_read.sum + dram__bytes_write.sum per launch divided by
# the launch's units) from one-kernel ncu captures of the network at 3/10 size:
#   ncu --set full --clock-control none -k regex:<kernel> -s <n> -c 2 python bench.py --scale 0.3 ...
# scaled to a full-size launch by its units
DELIVERY_TRAFFIC_PER_EVENT = 95.6e6 / 5.82e6   # bytes per synaptic event
RK5_TRAFFIC_PER_NEURON_STEP = 74.7e6 / 3.0e6   # bytes per neuron-step


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--scale", type=float, default=1.0, help="fraction of the 1M-neuron network (tests)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch mappings")
    p.add_argument("--mapping", default="",
                   help="fixed launch mapping instead of the autotuner: update threads, register-capped "
                        "variant (0/1/2), delivery lane group, delivery blocks, RK5 budget and optionally "
                        "programmatic launch (0/1), one RK5 trial per iteration (0/1), warp-aggregated "
                        "delivery (0/1) and pipelined delivery (0/1), e.g. 64,2,32,592,1")
    p.add_argument("--batch-max", type=int, default=0, help="upper bound of the time-batch length")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the learned-step and ensemble measurements")
    p.add_argument("--no-ref-cuda", action="store_true",
                   help="skip the timing of the reference's own CUDA build (several minutes)")
    p.add_argument("--partition", action="store_true",
                   help="with N > 1 GPUs: one 1M-neuron network split over the GPUs (spikes exchanged "
                        "over NCCL after every time batch, strong scaling) instead of one replica per GPU")
    return p.parse_args()


class ClockSampler(object):
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        sm.sort()
        loaded = [x for x in sm if mx and x > 0.5 * mx] or sm
        med = loaded[len(loaded) // 2] if loaded else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_engine_network(ngpu, scale, seed):
    from workloads import benchmark_network
    ngpu.SetVerbosityLevel(0)
    return benchmark_network(ngpu, scale, seed)


def ensemble_run(ngpu, bio_ms=1000.0):
    """256 independent networks (nest-gpu_b200/ensemble.py) advanced together; the launch
    mappings are autotuned first."""
    import numpy as np
    from ensemble import build_ensemble, ensemble_spec, ensemble_synapses, per_network_rates
    ngpu.Reset()
    ngpu.SetVerbosityLevel(0)
    spec = ensemble_spec()
    t0 = time.time()
    groups, layout = build_ensemble(ngpu, spec)
    ngpu.Calibrate()
    build_s = time.time() - t0
    t1 = time.time()
    chosen = ngpu.Autotune(200)
    tune_s = time.time() - t1
    ngpu.Simulate(100.0)
    counts0 = {m: np.asarray(ngpu.GetStatus(g, "spike_count")).ravel() for m, g in groups.items()}
    st0, l0 = ngpu.GetStats(), ngpu.GetLaunchCount()
    ngpu.Simulate(bio_ms)
    dev_s = ngpu.GetSimDeviceMs() / 1000.0
    st1, l1 = ngpu.GetStats(), ngpu.GetLaunchCount()
    rates, _ = per_network_rates(ngpu, groups, layout, counts0, bio_ms)
    n_neurons = int(sum(x["n"] for x in spec))
    # kernel time per step (each kernel bracketed by events) against the graph-timed step:
    # the difference bounds what a persistent launch could save over the captured graphs
    prof = ngpu.ProfileSteps(300)
    step_ms = dev_s * 1000.0 / (bio_ms / 0.1)
    out = {"networks": len(spec), "neurons": n_neurons, "synapses": ensemble_synapses(spec),
           "bio_ms": bio_ms, "rtf": dev_s / (bio_ms / 1000.0),
           "events_per_s": (st1["n_events"] - st0["n_events"]) / dev_s,
           "launches_per_step": (l1 - l0) / (bio_ms / 0.1),
           "rate_hz_min_median_max": [float(rates.min()), float(np.median(rates)), float(rates.max())],
           "mapping": chosen, "build_s": build_s, "autotune_s": tune_s,
           "ms_per_step": step_ms, "kernel_ms_per_step": sum(prof),
           "launch_gap_frac": max(0.0, 1.0 - sum(prof) / step_ms)}
    # the same networks one after another, each alone in the engine with its own graphs and
    # the default launch mapping: what batching them into one ensemble gains
    seq_ms, seq_bio = 0.0, 200.0
    t_seq = time.time()
    for net in spec:
        ngpu.Reset()
        ngpu.SetVerbosityLevel(0)
        build_ensemble(ngpu, [net])
        ngpu.Calibrate()
        ngpu.Simulate(20.0)
        ngpu.Simulate(seq_bio)
        seq_ms += ngpu.GetSimDeviceMs()
    out["sequential_rtf"] = (seq_ms / 1000.0) / (seq_bio / 1000.0)
    out["sequential_bio_ms_per_network"] = seq_bio
    out["sequential_wall_s"] = time.time() - t_seq
    out["batching_gain"] = out["sequential_rtf"] / out["rtf"]
    ngpu.Reset()
    return out


def ref_cuda_leg(args):
    """The reference's own CUDA build (oracle/_ref/libnestgpukernel.so, compiled from the
    reference sources) on this GPU, through the same nestgpu.py interface in child processes
    (tests/ref_runner.py; the reference keeps one network per process):
      - the benchmark network, identical edges (the generated blocks as edge lists), 500 ms
        first call, then 1000 ms timed as the reference's own "Simulation time" (wall time of
        Simulate, src/nestgpu.cu:458-463);
      - the microcircuit (workloads.microcircuit) through both libraries, same protocol."""
    lib = os.path.join(HERE, "oracle", "_ref", "libnestgpukernel.so")
    if not os.path.exists(lib):
        return {"unavailable": "reference library not built (oracle/Makefile.ref)"}
    runner = os.path.join(HERE, "tests", "ref_runner.py")

    def child(what, ref, extra_env=None, timeout=1500):
        env = dict(os.environ)
        env.pop("NESTGPU_LIB", None)
        if ref:
            env["NESTGPU_LIB"] = lib
        env.update(extra_env or {})
        p = subprocess.run([sys.executable, runner, what], env=env, capture_output=True, text=True,
                           timeout=timeout)
        if p.returncode != 0:
            return {"error": p.stderr[-500:]}
        return json.loads([x for x in p.stdout.splitlines() if x.startswith("JSON:")][-1][5:])

    out = {"library": "oracle/_ref/libnestgpukernel.so (reference sources, nvcc 12.9, sm_100, maxrregcount 55)",
           "protocol": "500 ms first call, then Simulate(1000) wall time, child process per run"}
    out["network_1M"] = child("timing_gen:%g:500:1000" % args.scale, True)
    out["microcircuit"] = child("microcircuit:1.0:1000:500", True)
    out["microcircuit_engine"] = child("microcircuit:1.0:1000:500", False, {"NGPU_AUTOTUNE": "1"})
    return out


def rank_reducers(dist, device):
    """Barrier and max / sum of one scalar over the ranks (identities without a process
    group); the only cross-rank traffic of the replicas."""
    def barrier():
        if dist is not None:
            dist.barrier()

    def reduce(x, op):
        if dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(x):
        return reduce(x, dist.ReduceOp.MAX) if dist is not None else x

    def sum_over_ranks(x):
        return reduce(x, dist.ReduceOp.SUM) if dist is not None else x

    return barrier, max_over_ranks, sum_over_ranks


def engine_arm(args):
    if WORLD > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(LOCAL_RANK)
    sys.path.insert(0, os.path.join(HERE, "nest-gpu_b200"))
    import numpy as np
    import nestgpu as ngpu
    dist = None
    if WORLD > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = tdist

    barrier, max_over_ranks, sum_over_ranks = rank_reducers(dist, "cuda")

    partitioned = args.partition and WORLD > 1
    seed = 20240 if partitioned else 20240 + 101 * RANK
    t_build0 = time.time()
    if args.batch_max > 0:
        ngpu.SetBatchMax(args.batch_max)
    neuron, pg = build_engine_network(ngpu, args.scale, seed)
    if partitioned:
        # every rank built the same network; it simulates its share and exchanges spikes
        from partition import TorchExchange
        exchange = TorchExchange(cap=1 << 18)
        exchange.attach()
    ngpu.Calibrate()
    build_s = time.time() - t_build0
    # launch mappings picked on this network (the trial steps are part of the transient)
    t_tune0 = time.time()
    if args.mapping:
        vals = [int(x) for x in args.mapping.split(",")]
        th, occ, grp, blk, bud = vals[:5]
        if len(vals) > 5:
            ngpu.SetProgrammaticLaunch(vals[5])
        if len(vals) > 6:
            ngpu.SetUpdateTrialIter(vals[6])
        if len(vals) > 7:
            ngpu.SetDeliverAggregate(vals[7])
        if len(vals) > 8:
            ngpu.SetDeliverPrefetch(vals[8])
        ngpu.SetUpdateThreads(th)
        ngpu.SetUpdateOccupancy(occ)
        ngpu.SetDeliverGroup(grp)
        ngpu.SetDeliverBlocks(blk)
        ngpu.SetRk5Budget(bud)
        mapping = ngpu.GetLaunchMapping()
    else:
        mapping = ngpu.Autotune(400) if not args.no_autotune else None
    tune_s = time.time() - t_tune0
    n_neurons = len(neuron)

    for _ in range(args.warmup):
        ngpu.Simulate(STEP_MS)
    st0 = ngpu.GetStats()
    l0 = ngpu.GetLaunchCount()
    sampler = ClockSampler(LOCAL_RANK)
    barrier()
    sampler.start()
    dev_ms = 0.0
    wall0 = time.time()
    for _ in range(args.steps):
        ngpu.Simulate(STEP_MS)
        dev_ms += ngpu.GetSimDeviceMs()
    wall = time.time() - wall0
    clocks = sampler.stop()
    barrier()
    st1 = ngpu.GetStats()
    launches = ngpu.GetLaunchCount() - l0
    events = st1["n_events"] - st0["n_events"]
    derivs = st1["n_derivs"] - st0["n_derivs"]
    spikes = st1["n_spikes"] - st0["n_spikes"]
    bio_s = args.steps * STEP_MS / 1000.0
    t_max = max_over_ranks(dev_ms / 1000.0)
    events_all = sum_over_ranks(float(events))
    value = events_all / t_max
    rtf = (dev_ms / 1000.0) / bio_s
    if partitioned:
        # each rank counted its own neurons' work; the network is the sum
        derivs = sum_over_ranks(float(derivs))
        spikes = sum_over_ranks(float(spikes))
        rtf = t_max / bio_s
    evals_per_neuron_ms = derivs / (n_neurons * args.steps * STEP_MS)
    rate_hz = spikes / (n_neurons * bio_s)

    # per-kernel device times (ordinary steps, each kernel bracketed by CUDA events)
    prof_steps = 200
    st_p0 = ngpu.GetStats()
    upd_ms, rec_ms, del_ms = ngpu.ProfileSteps(prof_steps)
    st_p1 = ngpu.GetStats()
    p_derivs = (st_p1["n_derivs"] - st_p0["n_derivs"]) / prof_steps
    p_events = (st_p1["n_events"] - st_p0["n_events"]) / prof_steps
    p_spikes = (st_p1["n_spikes"] - st_p0["n_spikes"]) / prof_steps
    M = ngpu.GetBatchLength()   # steps per launch of the update and delivery kernels
    fp32_peak = (148 * 128 * 2 * (clocks["sm_mhz"] or 1965.0) * 1e6) / 1e12
    rk5_tflops = p_derivs * FLOPS_PER_DERIV / (upd_ms / 1e3) / 1e12
    deliver_gbs = (p_events * DELIVERY_BYTES_PER_EVENT + p_spikes * DELIVERY_BYTES_PER_SPIKE) / (del_ms / 1e3) / 1e9
    # each synaptic event is one FP64 reduction into a random entry of one accumulator slot
    # (n_neurons x 2 receptor ports x 8 B): its measured random-reduction rate is the second
    # denominator of the delivery kernel
    red_gops = p_events / (del_ms / 1e3) / 1e9
    red_peak = ngpu.MeasureReductionRate(n_neurons * 2 * 8, 1 << 26)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    # end to end through the public API: per step a host->device parameter write, the
    # Simulate call and a device->host read of every neuron's spike count
    e2e_steps = max(1, args.steps)
    wall_e0 = time.time()
    ev_e0 = ngpu.GetStats()["n_events"]
    for _ in range(e2e_steps):
        ngpu.SetStatus(pg, "rate", PG_RATE)
        ngpu.Simulate(STEP_MS)
        counts = ngpu.GetSpikeCountArray(neuron)   # 4 MB device-to-host, as a NumPy array
    e2e_wall = time.time() - wall_e0
    e2e_events = ngpu.GetStats()["n_events"] - ev_e0
    e2e_t = max_over_ranks(e2e_wall)
    e2e_value = sum_over_ranks(float(e2e_events)) / e2e_t
    assert len(counts) == n_neurons

    result = {
        "metric": "synaptic events/s, 1M aeif_cond_beta_multisynapse x 1000 synapses (1e9), dt 0.1 ms",
        "value": value,
        "unit": "events/s",
        "n_gpus": WORLD,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max * 1000.0 / args.steps,
        "higher_is_better": True,
        "scaling": "strong" if partitioned else "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded random network and Poisson drive)",
        "config": {"workload": "1M aeif_cond_beta_multisynapse x 1000 synapses, Poisson 8 kHz, delays 1-2 ms", "neurons": n_neurons,
                   "synapses": n_neurons * (K_EXC + K_INH), "bio_ms_per_step": STEP_MS,
                   "dt_ms": 0.1,
                   "parallelism": ("partition%d" % WORLD) if partitioned else ("replicas%d" % WORLD),
                   "l2": "inputs larger than L2 (8 GB edge array)", "scale": args.scale},
        "rtf": rtf,
        "rk5_evals_per_neuron_ms": evals_per_neuron_ms,
        "firing_rate_hz": rate_hz,
        "build_s": build_s,
        "mapping": mapping,
        "autotune_s": tune_s,
        "gpu_launches": launches,
        "e2e": {"value": e2e_value, "unit": "events/s", "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 4 * n_neurons},
        "roofline": {"bound": "fp32", "kernel": "aeif_batch_kernel + aeif_straggler_kernel (RK5)",
                     "achieved": rk5_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": rk5_tflops / fp32_peak,
                     "traffic": RK5_TRAFFIC_PER_NEURON_STEP * n_neurons * M,
                     "flops_per_launch": p_derivs * FLOPS_PER_DERIV * M, "steps_per_launch": M,
                     "peak_source": "nominal FP32 rate 148 SM x 128 lanes x 2 x sampled SM clock",
                     "ms_per_step": upd_ms},
        "roofline_delivery": {"bound": "hbm", "kernel": "deliver_batch_kernel", "achieved": deliver_gbs,
                              "peak": hbm_peak, "unit": "GB/s", "frac": deliver_gbs / hbm_peak,
                              "traffic": DELIVERY_TRAFFIC_PER_EVENT * p_events * M,
                              "bytes_per_launch": (p_events * DELIVERY_BYTES_PER_EVENT +
                                                   p_spikes * DELIVERY_BYTES_PER_SPIKE) * M, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                              "ms_per_step": del_ms,
                              "reductions": {"achieved": red_gops, "peak": red_peak, "unit": "1e9 FP64 red/s",
                                             "frac": red_gops / red_peak,
                                             "peak_source": "measured in this run: random FP64 reductions into a "
                                                            "buffer of one accumulator slot's size"}},
        "clocks": clocks,
        # the per-kernel times above are CUDA-event brackets around each kernel of ordinary
        # steps (serialised, outside the graphs); their sum against the graph-timed step
        "kernel_timing": {"method": "CUDA events around each kernel (ProfileSteps), serialised",
                          "sum_ms_per_step": upd_ms + rec_ms + del_ms,
                          "graph_ms_per_step": dev_ms / (args.steps * STEP_MS / 0.1),
                          "sum_over_graph": (upd_ms + rec_ms + del_ms) / (dev_ms / (args.steps * STEP_MS / 0.1))},
    }
    if WORLD == 1 and not args.no_extras:
        from workloads import learned_vs_plain
        result["rk5_learned"] = [learned_vs_plain(ngpu, w) for w in (0.1, 1.0)]
        result["ensemble"] = ensemble_run(ngpu)
    if WORLD == 1 and not args.no_ref_cuda:
        rc = ref_cuda_leg(args)
        net = rc.get("network_1M", {})
        if "rtf" in net:
            rc["rtf_ratio"] = net["rtf"] / rtf                  # reference RTF / engine RTF
            rc["engine_rtf"] = rtf
            rc["engine_rate_hz"] = rate_hz
        mc, mce = rc.get("microcircuit", {}), rc.get("microcircuit_engine", {})
        if "rtf" in mc and "rtf" in mce:
            rc["rtf_ratio_microcircuit"] = mc["rtf"] / mce["rtf"]
        result["ref_cuda"] = rc
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_sample(steps=1, warmup=0)["cpu_baseline"]
    if RANK == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cpu_sample(steps, warmup):
    """CPU restatement (oracle, OpenMP) on a 20k-neuron sample of the workload."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import numpy as np
    import oracle as orc
    n = 20_000
    ne = int(0.8 * n)
    rng = np.random.RandomState(7)
    o = orc.Oracle(fp64=False)
    o.SetKernelStatus("rnd_seed", 7)
    neuron = o.Create("aeif_cond_beta_multisynapse", n, 2)
    o.SetStatus(neuron, {"E_rev": [0.0, -85.0]})
    pg = o.Create("poisson_generator")
    o.SetStatus(pg, "rate", PG_RATE)
    o.Connect(pg, neuron, {"rule": "all_to_all"}, {"weight": W_PG, "delay": 1.0, "receptor": 0})
    tgt = np.repeat(np.arange(n, dtype=np.int32), K_EXC + K_INH)
    src = np.concatenate([rng.randint(0, ne, size=(n, K_EXC)), rng.randint(ne, n, size=(n, K_INH))],
                         axis=1).astype(np.int32).ravel()
    port = np.tile(np.r_[np.zeros(K_EXC), np.ones(K_INH)].astype(np.int32), n)
    w = np.tile(np.r_[np.full(K_EXC, W_EXC), np.full(K_INH, W_INH)].astype(np.float32), n)
    d = (rng.randint(10, 21, size=src.size) * 0.1).astype(np.float32)
    o.ConnectArrays(src, tgt, port, w, d)
    o.ActivateSpikeCount(neuron)
    threads = o.Threads()
    for _ in range(warmup):
        o.Simulate(STEP_MS)
    e0, s0 = o.NEvents(), o.NSpikes()
    t0 = time.time()
    for _ in range(steps):
        o.Simulate(STEP_MS)
    dt = time.time() - t0
    ev = o.NEvents() - e0
    bio = steps * STEP_MS / 1000.0
    ev_s = ev / dt
    rate = (o.NSpikes() - s0) / n / bio
    rtf_full = (dt / bio) * (1_000_000 / n)
    return {"value": ev_s, "rtf_extrapolated_1M": rtf_full, "seconds": dt, "rate_hz": rate,
            "cpu_baseline": {"value": ev_s, "unit": "events/s", "cores": threads, "kind": "port",
                             "rate_hz": rate,
                             "sample": "20,000-neuron sample (same in-degree 800 + 200, drawn from the "
                                       "sample's 20k neurons; weights, delays, Poisson drive as the 1M "
                                       "network), %g ms bio per step, firing rate %.2f Hz (the 1M network: "
                                       "~16 Hz); RTF extrapolated to 1M neurons = %.1f"
                                       % (STEP_MS, rate, rtf_full)}}


def reference_arm(args):
    if RANK != 0:
        return
    r = cpu_sample(args.steps, args.warmup)
    out = {
        "impl": "reference",
        "metric": "synaptic events/s, 1M aeif_cond_beta_multisynapse x 1000 synapses (1e9), dt 0.1 ms",
        "value": r["value"],
        "unit": "events/s",
        "n_gpus": WORLD,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["seconds"] * 1000.0 / max(args.steps, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded random network and Poisson drive)",
        "config": {"workload": "1M aeif_cond_beta_multisynapse x 1000 synapses, Poisson 8 kHz, delays 1-2 ms", "sample_neurons": 20000,
                   "bio_ms_per_step": STEP_MS, "dt_ms": 0.1},
        "rtf_extrapolated_1M": r["rtf_extrapolated_1M"],
        "cpu_baseline": dict(r["cpu_baseline"]),
        "e2e": {"value": r["value"], "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
