// Learned RK5 step-size proposal: layout of the flat parameter vector, of the
// logged step tuples, and the feature definition, shared by the kernels and the
// host runtime.
//
// Features of a step (computed after its first derivative evaluation k1, with
// y the state at the step start):
//   f0 V_m, f1 w, f2..f5 the first state variable of ports 0..3 (g for the
//   conductance models, I_syn for the current models; 0 for missing ports),
//   f6 slog(dV_m/dt) (k1[0]), f7 slog of the sum over all ports of the derivative
//   of that variable, f8 log of the controller's h entering the step, f9 log of
//   the remaining interval (x1 - x); slog(x) = sign(x) log(1 + |x|).
// Network: xn = clamp((f - mu) * inv_sigma, -8, 8); a1 = relu(W1 xn + b1) (32);
// a2 = relu(W2 a1
// + b2) (32); out = W3 a2 + b3; the proposal is safety * exp(out * label_sigma +
// label_mu), raised to at least floor * (the controller's h) when floor > 0.
// Weights W1, W2, W3 are BF16 values (stored as floats whose low 16 bits are
// zero); biases and accumulation are FP32.
// Training target of a logged step: log(h_acc) - 0.2 * log(max(err, err_min)),
// the step size at which the embedded error estimate would reach the tolerance
// under the local h^5 error model.
#pragma once

namespace ngpu {

constexpr int SM_NF = 10;      // features
constexpr int SM_NH = 32;      // hidden width (both layers)
constexpr float SM_XCLAMP = 8.0f;   // normalised inputs are clamped to [-8, 8]

// flat parameter vector (floats)
constexpr int SM_MU = 0;
constexpr int SM_ISIG = SM_MU + SM_NF;
constexpr int SM_W1 = SM_ISIG + SM_NF;           // [NH][NF]
constexpr int SM_B1 = SM_W1 + SM_NH * SM_NF;
constexpr int SM_W2 = SM_B1 + SM_NH;             // [NH][NH]
constexpr int SM_B2 = SM_W2 + SM_NH * SM_NH;
constexpr int SM_W3 = SM_B2 + SM_NH;             // [NH]
constexpr int SM_B3 = SM_W3 + SM_NH;
constexpr int SM_LMU = SM_B3 + 1;
constexpr int SM_LSIG = SM_LMU + 1;
constexpr int SM_SAFETY = SM_LSIG + 1;
constexpr int SM_FLOOR = SM_SAFETY + 1;          // proposal >= floor * controller h (0: no floor)
constexpr int SM_NPAR = SM_FLOOR + 1;            // 1465
// trainable block W1 .. b3
constexpr int SM_TRAIN0 = SM_W1;
constexpr int SM_NTRAIN = SM_B3 + 1 - SM_W1;     // 1441

// logged tuple: features, accepted h, error of the accepted trial
constexpr int LOG_W = SM_NF + 2;

// LM_BOUND: analysis mode, every step starts from the largest step that passes the error
// test (the floor of evaluations any proposal can reach; the search is not counted)
enum LearnMode { LM_PLAIN = 0, LM_LOG = 1, LM_PROPOSE = 2, LM_BOUND = 3 };

}  // namespace ngpu
