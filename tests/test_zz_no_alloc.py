"""The allocation-free packing entry point against the allocating one.

NGPU_BuildDeliveryCsrNoAlloc exists for callers that may not call cudaMalloc (a
PyTorch program whose caching allocator owns the device heap, or a service that
splits each GPU into fixed pools at start-up): it takes its scratch from a static
device array inside the library.  Its results must equal NGPU_BuildDeliveryCsr's:
identical segment offsets and, inside every segment, the same edges (the order
inside a segment is unspecified for both).  Two calls in a row share the array,
so the second also checks that each call clears what it reuses.  This file is
named to run last; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import nestgpu as ngpu

pytestmark = pytest.mark.gpu


def bind(name):
    f = getattr(ngpu._lib, name)
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def device_edges(n, n_nodes, dspan, seed):
    import torch
    rng = np.random.RandomState(seed)
    dev = torch.device("cuda:0")
    src = torch.from_numpy(rng.randint(0, n_nodes, size=n).astype(np.int32)).to(dev)
    dly = torch.from_numpy(rng.randint(0, dspan, size=n).astype(np.int32)).to(dev)
    tgt = torch.from_numpy(rng.randint(0, 1 << 24, size=n).astype(np.int32)).to(dev)
    w = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(dev)
    return src, dly, tgt, w


def pack(fn, edges, n_nodes, dspan):
    import torch
    src, dly, tgt, w = edges
    n = src.numel()
    off = torch.full((n_nodes * dspan + 1,), -1, dtype=torch.int64, device=src.device)
    edge = torch.zeros(2 * max(n, 1), dtype=torch.int32, device=src.device)
    torch.cuda.synchronize()
    rc = fn(src.data_ptr(), dly.data_ptr(), tgt.data_ptr(), w.data_ptr(), n, n_nodes, dspan, off.data_ptr(),
            edge.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0, ngpu.GetErrorMessage()
    e = edge.cpu().numpy()[:2 * n].reshape(-1, 2)
    return off.cpu().numpy(), e[:, 0].copy(), e[:, 1].view(np.float32).copy()


def same_segments(a, b):
    off_a, t_a, w_a = a
    off_b, t_b, w_b = b
    assert np.array_equal(off_a, off_b)
    for s in range(off_a.size - 1):
        lo, hi = int(off_a[s]), int(off_a[s + 1])
        if hi - lo > 1:
            ka = sorted(zip(t_a[lo:hi].tolist(), w_a[lo:hi].tolist()))
            kb = sorted(zip(t_b[lo:hi].tolist(), w_b[lo:hi].tolist()))
            assert ka == kb, s
        elif hi - lo == 1:
            assert t_a[lo] == t_b[lo] and w_a[lo] == w_b[lo]


def test_noalloc_matches_allocating_entry_point_twice():
    alloc = bind("NGPU_BuildDeliveryCsr")
    noalloc = bind("NGPU_BuildDeliveryCsrNoAlloc")
    cases = [(300_000, 20_000, 11, 1), (50_000, 4_000, 25, 2)]
    for n, n_nodes, dspan, seed in cases:
        edges = device_edges(n, n_nodes, dspan, seed)
        ref = pack(alloc, edges, n_nodes, dspan)
        first = pack(noalloc, edges, n_nodes, dspan)
        second = pack(noalloc, edges, n_nodes, dspan)
        same_segments(ref, first)
        same_segments(ref, second)
        assert int(ref[0][-1]) == n


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    noalloc = bind("NGPU_BuildDeliveryCsrNoAlloc")
    edges = device_edges(10, 600_000, 1, 3)
    src, dly, tgt, w = edges
    off = torch.zeros(600_001, dtype=torch.int64, device=src.device)
    edge = torch.zeros(20, dtype=torch.int32, device=src.device)
    rc = noalloc(src.data_ptr(), dly.data_ptr(), tgt.data_ptr(), w.data_ptr(), 10, 600_000, 1, off.data_ptr(),
                 edge.data_ptr(), None)
    assert rc == -1 and ngpu.GetErrorCode() == 2
    assert "segments" in ngpu.GetErrorMessage()


def test_noalloc_reports_out_of_range_index_then_recovers():
    """A source or delay index outside the declared ranges is reported through the shared
    status word of the scratch array; the next valid call starts from a cleared word and
    packs like the allocating entry point."""
    import torch
    alloc = bind("NGPU_BuildDeliveryCsr")
    noalloc = bind("NGPU_BuildDeliveryCsrNoAlloc")
    n_nodes, dspan = 3000, 7
    for field, bad_value in ((0, n_nodes), (1, dspan)):
        edges = list(device_edges(20_000, n_nodes, dspan, 4 + field))
        bad = edges[field].clone()
        bad[123] = bad_value
        off = torch.zeros(n_nodes * dspan + 1, dtype=torch.int64, device=bad.device)
        edge = torch.zeros(2 * 20_000, dtype=torch.int32, device=bad.device)
        args = [x.data_ptr() for x in (edges[0], edges[1], edges[2], edges[3])]
        args[field] = bad.data_ptr()
        torch.cuda.synchronize()
        rc = noalloc(*args, 20_000, n_nodes, dspan, off.data_ptr(), edge.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == -1 and ngpu.GetErrorCode() != 0
        assert "out of range" in ngpu.GetErrorMessage()
        ref = pack(alloc, edges, n_nodes, dspan)
        again = pack(noalloc, edges, n_nodes, dspan)
        same_segments(ref, again)
