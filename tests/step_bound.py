"""Floor of RK5 derivative evaluations for any step-size proposal on the four-receptor
balanced network, computed with the oracle.

In bound mode every RK5 step starts from the largest step that passes the unchanged error
test (bisection), so no proposal, learned or not, can need fewer evaluations while keeping
the reference's accept/reject rule.  Prints plain vs bound evaluations per neuron-ms.

    python tests/step_bound.py [seed] [drive_nS ...]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "nest-gpu_b200"))

import numpy as np  # noqa: E402

import oracle as orc  # noqa: E402
from workloads import c4_network  # noqa: E402


def evals(seed, drive_w, bound, warm_ms=100.0, t_ms=500.0):
    o = orc.Oracle()
    n = c4_network(o, seed, drive_w=drive_w)
    o.Simulate(warm_ms)
    if bound:
        o.StepBoundMode(True)
    d0 = o.NDerivs()
    c0 = np.asarray(o.GetStatus(n, "spike_count")).sum()
    o.Simulate(t_ms)
    c1 = np.asarray(o.GetStatus(n, "spike_count")).sum()
    return (o.NDerivs() - d0) / (len(n) * t_ms), (c1 - c0) / len(n) / (t_ms / 1000.0)


def main():
    seed = int(sys.argv[1]) if len(sys.argv) > 1 else 43
    drives = [float(x) for x in sys.argv[2:]] or [0.1, 0.5, 1.0]
    for w in drives:
        p, rp = evals(seed, w, False)
        b, rb = evals(seed, w, True)
        print("seed %d drive %.2f nS: plain %.3f evals/neuron-ms (%.2f Hz), bound %.3f (%.2f Hz), "
              "largest possible reduction x%.3f" % (seed, w, p, rp, b, rb, p / b), flush=True)


if __name__ == "__main__":
    main()
