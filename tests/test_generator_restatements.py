"""The generated fixed in-degree rule behind the benchmark networks, three ways.

The engine draws the per-target sources and delays of ConnectFixedIndegreeGPU on the
device; the oracle restates the rule in C++ (oracle/ngpu_oracle.cpp, connect_generated);
tests/ref_runner.py restates it in numpy to feed the identical network to the reference
library as edge lists.  Here the numpy restatement is checked against the oracle edge by
edge (the GPU side is checked against the oracle in test_gpu_pinned.py).
"""
import numpy as np

import oracle as orc
from ref_runner import generated_edges, philox4x32_10
from workloads import benchmark_network


def test_philox_known_answer():
    # Philox4x32-10 known-answer vectors (Salmon et al. 2011, Random123 kat_vectors)
    x = philox4x32_10(0, 0, 0, 0, 0, 0)
    assert [int(v) for v in x] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    x = philox4x32_10(0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF)
    assert [int(v) for v in x] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def test_numpy_generator_equals_oracle():
    o = orc.Oracle()
    neuron, pg = benchmark_network(o, 0.002, 20240)     # 2000 neurons, 2e6 synapses
    c = o.ConnectionArrays()
    keep = c["source"] != pg[0]
    src, tgt, port = c["source"][keep], c["target"][keep], c["port"][keep]
    step = np.round(c["delay"][keep] / np.float32(0.1)).astype(np.int64) - 1
    n = len(neuron)
    n_exc = int(0.8 * n)
    for p, (s0, ns, k, seed) in enumerate(((0, n_exc, 800, 20240), (n_exc, n - n_exc, 200, 20240 + 7919))):
        t, s, d = generated_edges(0, n, k, ns, 11, seed)
        m = port == p
        exp = np.lexsort((d + 9, s + s0, t))
        got = np.lexsort((step[m], src[m], tgt[m]))
        assert np.array_equal((t + neuron.i0)[exp], tgt[m][got])
        assert np.array_equal((s + s0 + neuron.i0)[exp], src[m][got])
        assert np.array_equal((d + 9)[exp], step[m][got])
