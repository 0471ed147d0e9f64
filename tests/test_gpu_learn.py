"""Learned RK5 step-size proposal on the GPU, against the oracle.

- the inference code (the same device function the RK5 kernels call) is bit-identical
  to the oracle's FP32 statement of the network;
- the training kernels' gradient (tensor-core products of BF16 operands, FP32 sums)
  agrees with the oracle's gradient at the same operand precision;
- the step log of the plain integrator holds exactly the oracle's tuples;
- with a network proposing, the simulation is bit-identical to the oracle's;
- trained on a logged run, the network keeps the firing statistics and does not cost
  RK5 evaluations on a held-out seed (the evaluation counts are printed)."""
import numpy as np
import pytest

import nestgpu as ngpu
import oracle as orc
from workloads import learned_vs_plain
from test_oracle_learn import constant_model, random_params, small_c4

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fresh_engine():
    ngpu.Reset()
    yield
    ngpu.Reset()


def test_mlp_forward_bit_exact():
    for seed in (1, 2):
        p = random_params(seed)
        f = np.random.RandomState(seed + 10).randn(3000, 10).astype(np.float32) * 2.0
        assert np.array_equal(ngpu.MlpForward(p, f), orc.mlp_out(p, f))


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 4099])
def test_mlp_gradient_vs_fp64_oracle(n):
    """The tensor-core kernel against the oracle with the same BF16 operand roundings (FP64
    sums; what remains is FP32 accumulation and, rarely, one BF16 rounding step of a value
    whose FP32 and FP64 forms straddle a rounding boundary), and against the unrounded FP64
    gradient at BF16 operand precision."""
    p = random_params(7)
    rng = np.random.RandomState(n)
    f = rng.randn(n, 10).astype(np.float32)
    t = rng.uniform(-7, -2, n).astype(np.float32)
    loss, g = ngpu.MlpGrad(p, f, t)
    loss_b, g_b = orc.mlp_grad_bf16(p, f, t)
    loss64, g64 = orc.mlp_grad(p, f, t)
    assert abs(loss - loss_b) <= 1e-4 * max(1.0, loss_b)
    scale = np.abs(g_b).max()
    assert np.max(np.abs(g.astype(np.float64) - g_b)) <= 5e-3 * scale + 1e-8
    assert np.median(np.abs(g.astype(np.float64) - g_b)) <= 1e-5 * scale + 1e-9
    assert abs(loss - loss64) <= 2e-2 * max(1.0, loss64)
    assert np.max(np.abs(g.astype(np.float64) - g64)) <= 5e-2 * np.abs(g64).max() + 1e-8


def test_mlp_gradient_wait_timeout_is_reported():
    """Failure path of the tensor-core training kernel: with the completion of its products
    never signalled, the bounded wait runs out, the call fails with an error instead of
    hanging, and the next call (hook off) is correct."""
    p = random_params(7)
    rng = np.random.RandomState(3)
    f = rng.randn(300, 10).astype(np.float32)
    t = rng.uniform(-7, -2, 300).astype(np.float32)
    ngpu._c["NGPU_TestTensorWaitTimeout"](1)
    try:
        with pytest.raises(ValueError, match="did not complete"):
            ngpu.MlpGrad(p, f, t)
    finally:
        ngpu._c["NGPU_TestTensorWaitTimeout"](0)
    loss, g = ngpu.MlpGrad(p, f, t)
    loss_b, g_b = orc.mlp_grad_bf16(p, f, t)
    assert abs(loss - loss_b) <= 1e-4 * max(1.0, loss_b)
    assert np.max(np.abs(g.astype(np.float64) - g_b)) <= 5e-3 * np.abs(g_b).max() + 1e-8


def sorted_rows(a):
    return a[np.lexsort(a.T[::-1])]


def test_step_log_matches_oracle():
    o = orc.Oracle()
    small_c4(o)
    small_c4(ngpu)
    for api in (o, ngpu):
        api.Simulate(10.0)
    o.Rk5LogStart(5_000_000)
    ngpu.Rk5LogStart(5_000_000)
    o.Simulate(20.0)
    ngpu.Simulate(20.0)
    o.Rk5LogStop()
    ngpu.Rk5LogStop()
    n_o, off_o = o.Rk5LogCount()
    n_g, off_g = ngpu.Rk5LogCount()
    assert n_o == n_g == off_o == off_g and n_g > 0
    a = sorted_rows(o.Rk5LogGet())
    b = sorted_rows(ngpu.Rk5LogGet())
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("which", ["constant", "random"])
def test_learned_proposal_bit_exact(which):
    if which == "constant":
        p = constant_model(0.013)
    else:
        p = random_params(21)
        p[1461], p[1462] = np.float32(np.log(0.02)), 0.5
    res = []
    for api in (orc.Oracle(), ngpu):
        n = small_c4(api, seed=5, drive_w=1.5)
        rec = api.CreateRecord("", ["V_m", "w", "g", "g1"], [n[0], n[3], n[7], n[9]], [0, 0, 1, 2])
        api.Simulate(5.0)
        if api is ngpu:
            ngpu.StepModelSet(p)
            ngpu.StepModelEnable(True)
        else:
            api.StepModelSet(p, enable=True)
        api.Simulate(25.0)
        counts = np.array(api.GetStatus(n, "spike_count")).ravel()
        nd = api.NDerivs() if api is not ngpu else ngpu.GetStats()["n_derivs"]
        res.append((counts, np.asarray(api.GetRecordData(rec), dtype=np.float32), nd))
    (c_o, r_o, nd_o), (c_g, r_g, nd_g) = res
    assert c_o.sum() > 0
    assert np.array_equal(c_o, c_g)
    assert np.array_equal(r_o.view(np.uint32), r_g.view(np.uint32))
    assert nd_o == nd_g


@pytest.mark.parametrize("drive_w", [0.1, 1.0])
def test_trained_proposal_on_held_out_seed(drive_w):
    """Log 2 s of the plain integrator, train on the GPU, pick the safety factor on the
    training seed, evaluate on a held-out seed: the proposal must not cost evaluations and
    must keep the firing rate, in the quiet network (0.1 nS drive) and the firing one."""
    r = learned_vs_plain(ngpu, drive_w, target_tuples=20_000_000, max_log_ms=4000.0)
    print("\nfour-receptor network, drive %.2f nS: %s" % (drive_w, r))
    assert abs(r["learned_rate_hz"] - r["plain_rate_hz"]) <= 0.02 * max(r["plain_rate_hz"], 1.0)
    assert r["logged_steps"] > 0 and r["trained_on"] > 0
    assert r["learned_evals_per_neuron_ms"] <= r["plain_evals_per_neuron_ms"]
    # the floor (every step from the largest passing step) is below both
    assert r["floor_evals_per_neuron_ms"] <= r["learned_evals_per_neuron_ms"]
    if drive_w == 1.0:
        # the firing network: the measured gain is 1.21x of a possible 1.34x; hold it above 1.15x
        assert r["ratio"] >= 1.15


def test_bound_mode_matches_oracle():
    """The floor measurement (every RK5 step starts from the largest step that passes the
    error test, found by bisection) gives the same evaluation count, spikes and traces on the
    GPU as the oracle's bound mode."""
    res = []
    for api in (orc.Oracle(), ngpu):
        n = small_c4(api, seed=5, drive_w=1.5)
        rec = api.CreateRecord("", ["V_m", "w"], [n[0], n[3]], [0, 0])
        api.Simulate(5.0)
        if api is ngpu:
            ngpu.StepBoundMode(True)
            d0 = ngpu.GetStats()["n_derivs"]
        else:
            api.StepBoundMode(True)
            d0 = api.NDerivs()
        api.Simulate(20.0)
        nd = (ngpu.GetStats()["n_derivs"] if api is ngpu else api.NDerivs()) - d0
        counts = np.array(api.GetStatus(n, "spike_count")).ravel()
        res.append((counts, np.asarray(api.GetRecordData(rec), dtype=np.float32), nd))
    (c_o, r_o, nd_o), (c_g, r_g, nd_g) = res
    assert c_o.sum() > 0
    assert np.array_equal(c_o, c_g)
    assert np.array_equal(r_o.view(np.uint32), r_g.view(np.uint32))
    assert nd_o == nd_g
