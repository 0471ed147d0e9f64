"""NGPU_BuildDeliveryCsr: device edge list -> (source, delay) segments, checked against a
numpy counting sort.  Device buffers come from torch; the entry point gets raw pointers."""
import ctypes

import numpy as np
import pytest

import nestgpu as ngpu

pytestmark = pytest.mark.gpu


def bind():
    f = ngpu._lib.NGPU_BuildDeliveryCsr
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def make_edges(n, n_nodes, dspan, seed):
    rng = np.random.RandomState(seed)
    src = rng.randint(0, n_nodes, size=n).astype(np.int32)
    dly = rng.randint(0, dspan, size=n).astype(np.int32)
    tgt = rng.randint(0, 1 << 20, size=n).astype(np.uint32)
    w = rng.standard_normal(n).astype(np.float32)
    return src, dly, tgt, w


def expected(src, dly, tgt, w, n_nodes, dspan):
    key = src.astype(np.int64) * dspan + dly
    cnt = np.bincount(key, minlength=n_nodes * dspan)
    off = np.zeros(n_nodes * dspan + 1, dtype=np.uint64)
    off[1:] = np.cumsum(cnt)
    return key, off


def run_pack(fn, src, dly, tgt, w, n_nodes, dspan):
    import torch
    dev = torch.device("cuda:0")
    t_src = torch.from_numpy(src).to(dev)
    t_dly = torch.from_numpy(dly).to(dev)
    t_tgt = torch.from_numpy(tgt.view(np.int32)).to(dev)
    t_w = torch.from_numpy(w).to(dev)
    off = torch.zeros(n_nodes * dspan + 1, dtype=torch.int64, device=dev)
    edge = torch.zeros(2 * src.size, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = fn(t_src.data_ptr(), t_dly.data_ptr(), t_tgt.data_ptr(), t_w.data_ptr(), src.size, n_nodes, dspan,
            off.data_ptr(), edge.data_ptr(), None)
    torch.cuda.synchronize()
    e = edge.cpu().numpy().reshape(-1, 2)
    return rc, off.cpu().numpy().view(np.uint64), e[:, 0].view(np.uint32), e[:, 1].view(np.float32)


def check_segments(off, key, tgt, w, g_off, g_tgt, g_w):
    assert np.array_equal(off, g_off)
    order = np.argsort(key, kind="stable")
    for s in np.nonzero(np.diff(off.astype(np.int64)))[0][:2000]:
        a, b = int(off[s]), int(off[s + 1])
        exp = sorted(zip(tgt[order[a:b]].tolist(), w[order[a:b]].tolist()))
        got = sorted(zip(g_tgt[a:b].tolist(), g_w[a:b].tolist()))
        assert exp == got


@pytest.mark.parametrize("n,n_nodes,dspan", [(0, 10, 3), (1, 1, 1), (100_000, 3000, 11),
                                             (2_000_000, 50_000, 20)])
def test_pack_matches_counting_sort(n, n_nodes, dspan):
    fn = bind()
    src, dly, tgt, w = make_edges(n, n_nodes, dspan, seed=n + dspan)
    key, off = expected(src, dly, tgt, w, n_nodes, dspan)
    rc, g_off, g_tgt, g_w = run_pack(fn, src, dly, tgt, w, n_nodes, dspan)
    assert rc == 0
    check_segments(off, key, tgt, w, g_off, g_tgt, g_w)


def test_pack_rejects_out_of_range_index():
    fn = bind()
    src, dly, tgt, w = make_edges(1000, 100, 4, seed=1)
    src[17] = 100
    rc, _, _, _ = run_pack(fn, src, dly, tgt, w, 100, 4)
    assert rc == -1 and ngpu.GetErrorCode() != 0
    assert "out of range" in ngpu.GetErrorMessage()
