"""The oracle's statement of the learned RK5 step-size proposal (no reference
counterpart): the 10-32-32-1 network, its FP64 gradient, the step-tuple log of the
plain integrator, and the proposal inside the RK5 loop.

The gradient is pinned by central finite differences of an independent numpy
float64 forward pass; the FP32 forward (the engine kernel's arithmetic) by that
same numpy pass within FP32 rounding."""
import numpy as np
import pytest

import oracle as orc
from scenarios import c4_network

NP, NT, T0 = orc.STEP_MODEL_NPAR, orc.STEP_MODEL_NTRAIN, orc.STEP_MODEL_TRAIN0
W1, B1, W2, B2, W3, B3, LMU, LSIG, SAF = 20, 340, 372, 1396, 1428, 1460, 1461, 1462, 1463


def bf16(a):
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def random_params(seed):
    rng = np.random.RandomState(seed)
    p = np.zeros(NP, dtype=np.float32)
    p[0:10] = rng.randn(10)
    p[10:20] = rng.uniform(0.5, 2.0, 10)
    p[W1:B1] = bf16(rng.randn(B1 - W1) * 0.5)
    p[B1:W2] = rng.randn(W2 - B1) * 0.1
    p[W2:B2] = bf16(rng.randn(B2 - W2) * 0.25)
    p[B2:W3] = rng.randn(W3 - B2) * 0.1
    p[W3:B3] = bf16(rng.randn(B3 - W3) * 0.3)
    p[B3] = 0.05
    p[LMU], p[LSIG], p[SAF] = -3.0, 1.5, 0.9
    return p


def np_forward(theta, p, f):
    """float64 forward with the trainable block taken from theta (float64)."""
    w1 = theta[0:320].reshape(32, 10)
    b1 = theta[320:352]
    w2 = theta[352:1376].reshape(32, 32)
    b2 = theta[1376:1408]
    w3 = theta[1408:1440]
    b3 = theta[1440]
    xn = np.clip((f.astype(np.float32) - p[0:10]) * p[10:20], -8.0, 8.0).astype(np.float64)
    a1 = np.maximum(xn @ w1.T + b1, 0.0)
    a2 = np.maximum(a1 @ w2.T + b2, 0.0)
    return a2 @ w3 + b3


def np_loss(theta, p, f, t):
    tn = (t.astype(np.float64) - p[LMU]) / np.float64(p[LSIG])
    r = np_forward(theta, p, f) - tn
    return np.mean(r * r)


def test_mlp_gradient_matches_finite_differences():
    p = random_params(3)
    rng = np.random.RandomState(4)
    f = rng.randn(64, 10).astype(np.float32)
    t = rng.uniform(-6, -1, 64).astype(np.float32)
    loss, g = orc.mlp_grad(p, f, t)
    theta = p[T0:T0 + NT].astype(np.float64)
    assert abs(loss - np_loss(theta, p, f, t)) <= 1e-12 * max(1.0, loss)
    idx = np.concatenate([rng.choice(NT, 80, replace=False), [0, 319, 320, 351, 352, 1375, 1376, 1407,
                                                             1408, 1439, 1440]])
    eps = 1e-6
    for j in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[j] += eps
        tm[j] -= eps
        num = (np_loss(tp, p, f, t) - np_loss(tm, p, f, t)) / (2 * eps)
        assert abs(num - g[j]) <= 1e-6 * max(1.0, np.abs(g).max()), (j, num, g[j])


def test_bf16_operand_gradient_restatement():
    """The oracle's statement of the GPU training kernel's operand precision (BF16 roundings
    of the values that enter the tensor-core products) stays within BF16 precision of the
    exact gradient, and equals it where every operand is already a BF16 value."""
    p = random_params(3)
    rng = np.random.RandomState(8)
    f = rng.randn(300, 10).astype(np.float32)
    t = rng.uniform(-6, -1, 300).astype(np.float32)
    loss, g = orc.mlp_grad(p, f, t)
    loss_b, g_b = orc.mlp_grad_bf16(p, f, t)
    assert abs(loss - loss_b) <= 1e-2 * max(1.0, loss)
    assert np.max(np.abs(g - g_b)) <= 5e-2 * np.abs(g).max()
    assert np.max(np.abs(g - g_b)) > 0.0
    # one sample whose normalised inputs are 0 and whose layer-1 units are all off: only the
    # output bias and its error remain, and d = 2 r is rounded to BF16 in the restatement
    q = p.copy()
    q[T0:T0 + NT] = 0.0
    q[B3] = 0.5
    q[B1:W2] = -1.0                                 # every layer-1 unit off
    f0 = np.zeros((1, 10), np.float32) + p[:10]    # inputs at the mean
    t0 = np.array([p[LMU]], np.float32)            # normalised target 0
    l0, g0 = orc.mlp_grad(q, f0, t0)
    l0b, g0b = orc.mlp_grad_bf16(q, f0, t0)
    assert l0 == l0b == 0.25
    assert g0[-1] == g0b[-1] == 1.0
    assert np.count_nonzero(g0b[:-1]) == 0


def test_mlp_fp32_forward_close_to_fp64():
    p = random_params(5)
    f = np.random.RandomState(6).randn(500, 10).astype(np.float32)
    out32 = orc.mlp_out(p, f)
    out64 = np_forward(p[T0:T0 + NT].astype(np.float64), p, f)
    assert np.all(np.abs(out32 - out64) <= 2e-5 * (1.0 + np.abs(out64)))
    prop = orc.mlp_propose(p, f)
    ref = p[SAF] * np.exp(out64 * p[LSIG] + p[LMU])
    assert np.allclose(prop, ref, rtol=1e-4)


def small_c4(o, seed=7, drive_w=1.0):
    return c4_network(o, seed, n=200, drive_w=drive_w)


def test_step_log_records_every_accepted_step():
    o = orc.Oracle()
    n = small_c4(o)
    o.Simulate(20.0)
    steps0 = o.NRk5Steps()
    o.Rk5LogStart(10_000_000)
    o.Simulate(30.0)
    o.Rk5LogStop()
    o.Simulate(5.0)
    nlog, offered = o.Rk5LogCount()
    assert nlog == offered
    steps1 = o.NRk5Steps()
    log = o.Rk5LogGet()
    assert log.shape == (nlog, orc.LOG_W)
    # logged steps are those of the 30 ms window; the network fired in it
    assert nlog > 0
    assert nlog <= steps1 - steps0
    assert np.array(o.GetStatus(n, "spike_count")).sum() > 0
    h, err = log[:, 10], log[:, 11]
    hmin = 1e-4
    assert np.all((err <= 1.0) | (h <= hmin * 1.00001))
    hmax = np.exp(log[:, 9].astype(np.float64))
    assert np.all(h <= hmax * (1 + 1e-5))
    assert np.all(log[:, 8] <= np.log(0.1) + 1e-3 + 5 * np.log(5.0))
    # capacity: the log keeps the first `cap` tuples and counts the rest
    o2 = orc.Oracle()
    small_c4(o2)
    o2.Rk5LogStart(1000)
    o2.Simulate(10.0)
    n2, off2 = o2.Rk5LogCount()
    assert n2 == 1000 and off2 > 1000


def constant_model(h):
    """A network whose proposal is exactly h everywhere: zero weights, label_mu = log h."""
    p = np.zeros(NP, dtype=np.float32)
    p[10:20] = 1.0
    p[LMU] = np.float32(orc.log_m(h))
    p[LSIG] = 1.0
    p[SAF] = 1.0
    return p


def test_proposal_keeps_error_control():
    """With the proposal active, every accepted step still passes the unchanged error
    test, so the trajectory stays within the tolerance of the FP64 integration."""
    res = {}
    for mode in ("fp64", "plain", "const"):
        o = orc.Oracle(fp64=(mode == "fp64"))
        n = small_c4(o, seed=11, drive_w=1.5)
        rec = o.CreateRecord("", ["V_m"] * 4, [n[0], n[1], n[2], n[3]], [0] * 4)
        if mode == "const":
            o.StepModelSet(constant_model(0.013), enable=True)
        o.Simulate(40.0)
        res[mode] = (np.asarray(o.GetRecordData(rec))[:, 1:], np.array(o.GetStatus(n, "spike_count")).ravel(),
                     o.NDerivs())
    # the network fires; FP32 and FP64 trajectories separate slowly (chaotic regime), so the
    # traces are compared over the first 10 ms and the spike totals over the whole run
    v64, c64, _ = res["fp64"]
    assert c64.sum() > 100
    for mode in ("plain", "const"):
        v, c, nd = res[mode]
        assert abs(int(c.sum()) - int(c64.sum())) <= max(2, 0.02 * c64.sum())
        assert np.max(np.abs(v[:100] - v64[:100])) < 1e-3
    assert res["const"][2] != res["plain"][2]


def test_bound_mode_is_a_floor():
    """The bound mode starts every step from the largest step that passes the error test;
    no proposal, learned or constant, needs fewer derivative evaluations, and the dynamics
    stay those of the same network."""
    res = {}
    for mode in ("plain", "bound", "const"):
        o = orc.Oracle()
        n = small_c4(o, seed=11, drive_w=1.5)
        if mode == "bound":
            o.StepBoundMode(True)
        elif mode == "const":
            o.StepModelSet(constant_model(0.02), enable=True)
        o.Simulate(50.0)
        res[mode] = (o.NDerivs(), int(np.array(o.GetStatus(n, "spike_count")).sum()),
                     o.NRk5Trials() - o.NRk5Steps())
    assert res["bound"][0] < res["plain"][0] and res["bound"][0] < res["const"][0]
    assert res["bound"][2] == 0          # the bound never needs a rejected trial
    assert abs(res["bound"][1] - res["plain"][1]) <= 0.02 * res["plain"][1]


def test_step_bound_script_small():
    """tests/step_bound.py (the floor of RK5 evaluations behind the learned-step
    comparison) at a short window: the bound never needs more evaluations than plain."""
    from step_bound import evals
    p, rp = evals(43, 1.0, False, warm_ms=10.0, t_ms=10.0)
    b, rb = evals(43, 1.0, True, warm_ms=10.0, t_ms=10.0)
    assert 60.0 <= b <= p
