// CPU oracle for the NEST GPU hot path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the host, the algorithms of the reference's spiking
// engine so that the CUDA engine in nest-gpu_b200/ can be checked against it.
// Nothing in the product links, imports or calls this code; only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
//
// What it follows (paths relative to the NEST GPU 1.08 source tree):
//   adaptive Cash-Karp RK5 step / update  src/rk5.h:69-174, constants src/rk5.cu:35-72
//   aeif_cond_beta_multisynapse           src/aeif_cond_beta_multisynapse_kernel.h:165-226,
//                                         src/aeif_cond_beta_multisynapse.cu:37-99,120-172
//   aeif_cond_alpha_multisynapse          src/aeif_cond_alpha_multisynapse_kernel.h (same harness)
//   aeif_psc_exp_multisynapse             src/aeif_psc_exp_multisynapse_kernel.h
//   aeif_psc_alpha_multisynapse           src/aeif_psc_alpha_multisynapse_kernel.h
//   iaf_psc_exp                           src/iaf_psc_exp.cu:68-175, src/propagator_stability.cu:31-52
//   spike_generator                       src/spike_generator.cu:49-67,230-290
//   per-source spike queue                src/spike_buffer.cu:162-317 (PushSpike, SpikeBufferUpdate)
//   event list + FP64 input accumulation  src/send_spike.cu:45-58, src/get_spike.cu:60-166
//   poiss_gen direct drive                src/poiss_gen.cu:55-86, src/nestgpu.cu:1190-1226
//   connection store and rules            src/connect.cu:38-74, src/connect_rules.h:161-338,
//                                         src/connect_rules.cpp:274-322
//   RandomInt / RandomNormal(Clipped)     src/random.cu:8-76, src/nestgpu.cu:1135-1188
//   step order                            src/nestgpu.cu:294-635
//   parrot_neuron                         src/parrot_neuron.cu:60-130
//   dendritic delay of reverse spikes     src/spike_buffer.cu:162-190,247-317
//   synapse groups and STDP               src/syn_model.cu:43-56,136-152, src/stdp.cu:36-80,
//                                         src/test_syn_model.cu:35-50, src/get_spike.cu:85-95,
//                                         src/rev_spike.cu:46-130, src/nestgpu.cu:490-498,606-616
//
// Two arithmetic modes:
//   fp64 = 0  "FP32 mirror": float state, explicit fused multiply-adds, the
//             same own exp/log, reciprocal-multiply and Poisson sampler that the
//             CUDA kernels use, so that results are bit-identical to them;
//   fp64 = 1  double state and std::exp/std::pow, the reference formulas with
//             true divisions: the accuracy yardstick for the FP32 engine.
// The Poisson drive is drawn from Philox4x32-10 (Salmon et al., SC'11) keyed by
// (seed, direct-edge id, time index); the reference uses cuRAND XORWOW device
// states, which are not bit-comparable, so that stream is a deliberate break.
// Connectivity random numbers come from cuRAND's host generator
// (CURAND_RNG_PSEUDO_DEFAULT), the library the reference itself calls.

#include <curand.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

// --------------------------------------------------------------------------
// Own float exp / log (Cody-Waite reduction, Taylor / atanh series).
// --------------------------------------------------------------------------
static inline float as_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
static inline uint32_t as_uint(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

static float exp_m(float x) {
  if (!(x == x)) return x;                       // NaN
  if (x > 88.72283935546875f) return INFINITY;
  if (x < -103.972084045410156f) return 0.0f;
  float n = std::rint(x * 1.44269502162933349609f);
  float r = std::fmaf(n, -0.693145751953125f, x);
  r = std::fmaf(n, -1.428606765330187045e-06f, r);
  float p = 1.98412701e-04f;                     // 1/5040
  p = std::fmaf(p, r, 1.38888892e-03f);          // 1/720
  p = std::fmaf(p, r, 8.33333377e-03f);          // 1/120
  p = std::fmaf(p, r, 4.16666679e-02f);          // 1/24
  p = std::fmaf(p, r, 1.66666672e-01f);          // 1/6
  p = std::fmaf(p, r, 0.5f);
  p = std::fmaf(p, r, 1.0f);
  p = std::fmaf(p, r, 1.0f);
  int ni = (int)n;
  int n1 = ni / 2;
  int n2 = ni - n1;
  p = p * as_float((uint32_t)(n1 + 127) << 23);
  p = p * as_float((uint32_t)(n2 + 127) << 23);
  return p;
}

static float log_m(float x) {
  if (!(x > 0.0f)) return (x == 0.0f) ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  if (x < 1.17549435e-38f) { x = x * 16777216.0f; e = -24; }   // subnormal
  uint32_t b = as_uint(x);
  e += (int)((b >> 23) & 0xff) - 127;
  float m = as_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = 9.09090936e-02f;                     // 1/11
  q = std::fmaf(q, s2, 1.11111112e-01f);         // 1/9
  q = std::fmaf(q, s2, 1.42857149e-01f);         // 1/7
  q = std::fmaf(q, s2, 2.00000003e-01f);         // 1/5
  q = std::fmaf(q, s2, 3.33333343e-01f);         // 1/3
  q = std::fmaf(q, s2, 1.0f);
  float lm = (2.0f * s) * q;
  float fe = (float)e;
  return std::fmaf(fe, 0.693145751953125f, std::fmaf(fe, 1.428606765330187045e-06f, lm));
}

// --------------------------------------------------------------------------
// Philox4x32-10 and the Poisson sampler used for the poiss_gen drive.
// --------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };
static inline void mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}
static U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c.x, hi0, lo0);
    mulhilo(0xCD9E8D57u, c.z, hi1, lo1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}
static inline float u01(uint32_t r) { return ((float)(r >> 8) + 0.5f) * 5.96046448e-08f; }

// 1/k rounded to float (k = 1..64): the inversion multiplies by it.
static float inv_k(int k) { return (k <= 64) ? (float)(1.0 / k) : 1.0f / (float)k; }

// Sequential-search inversion from p(0) = emlam = exp(-lam).
static int poisson_small(float lam, float emlam, float u) {
  float p = emlam;
  float F = p;
  int k = 0;
  while (u > F && p > 9.31322575e-10f && k < 1000) {
    k++;
    p = (p * lam) * inv_k(k);
    F = F + p;
  }
  return k;
}

static uint32_t word_of(const U4 &r, int w) { return w == 0 ? r.x : w == 1 ? r.y : w == 2 ? r.z : r.w; }

// Philox block of edge `edge` for the time indices 4*(tidx/4) .. +3, chunk field j.
static U4 poisson_block(uint64_t seed, uint64_t edge, int64_t tidx, uint32_t j) {
  U4 c;
  c.x = (uint32_t)edge;
  c.y = (uint32_t)(edge >> 32);
  c.z = (uint32_t)((uint64_t)tidx >> 2);
  c.w = ((uint32_t)((uint64_t)tidx >> 34) & 0xffffu) | (j << 16);
  return philox(c, (uint32_t)seed ^ 0x6A09E667u, (uint32_t)(seed >> 32) ^ 0xBB67AE85u);
}

// n ~ Poisson(lam) for direct edge `edge` at time index `tidx`: word tidx % 4 of the
// edge's block for tidx / 4; lam > 10 is split into ceil(lam / 10) chunks (fields 1..).
static int poisson_draw(float lam, uint64_t seed, uint64_t edge, int64_t tidx) {
  if (!(lam > 0.0f)) return 0;
  const int w = (int)(tidx & 3);
  if (lam <= 10.0f) return poisson_small(lam, exp_m(-lam), u01(word_of(poisson_block(seed, edge, tidx, 0), w)));
  const int m = (int)std::ceil(lam / 10.0f);
  const float lc = lam / (float)m;
  const float emlc = exp_m(-lc);
  int n = 0;
  for (int j = 0; j < m; j++)
    n += poisson_small(lc, emlc, u01(word_of(poisson_block(seed, edge, tidx, (uint32_t)(j + 1)), w)));
  return n;
}

// --------------------------------------------------------------------------
// Models
// --------------------------------------------------------------------------
enum Model { AEIF_COND_BETA = 0, AEIF_COND_ALPHA, AEIF_PSC_EXP, AEIF_PSC_ALPHA,
             IAF_PSC_EXP, SPIKE_GEN, POISS_GEN, PARROT, SPIKE_DET, N_MODEL };

static const char *model_name[N_MODEL] = {
  "aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse",
  "aeif_psc_exp_multisynapse", "aeif_psc_alpha_multisynapse",
  "iaf_psc_exp", "spike_generator", "poisson_generator", "parrot_neuron", "spike_detector"};

// parrot_neuron (src/parrot_neuron.cu:40-52): port 0 input (weight 1) repeated as a spike in
// the next step, port 1 input weighted 0 (it only reaches plastic synapses)
enum { PR_input_spike_height = 0, PR_dummy_input, PR_V, PR_NVAR };
static const char *parrot_var_name[PR_NVAR] = {"input_spike_height", "dummy_input", "V"};
enum { PR_hold_spike_height = 0, PR_den_delay, PR_NPAR };
static const char *parrot_par_name[PR_NPAR] = {"hold_spike_height", "den_delay"};

// spike_detector (src/spike_detector.cu:28-70): the input of a step (one port, weight 1)
// becomes spike_height in the next one (1, or the input with hold_spike_height, default 1)
enum { SD_input_spike_height = 0, SD_spike_height, SD_NVAR };
static const char *sdet_var_name[SD_NVAR] = {"input_spike_height", "spike_height"};
enum { SD_hold_spike_height = 0, SD_NPAR };
static const char *sdet_par_name[SD_NPAR] = {"hold_spike_height"};

static bool is_aeif(Model m) { return m <= AEIF_PSC_ALPHA; }

// Scalar parameters of the aeif family (reference index order).
enum { A_V_th = 0, A_Delta_T, A_g_L, A_E_L, A_C_m, A_a, A_b, A_tau_w, A_I_e,
       A_V_peak, A_V_reset, A_t_ref, A_refractory_step, A_den_delay, A_NSCAL };
static const char *aeif_scal_name[A_NSCAL] = {
  "V_th", "Delta_T", "g_L", "E_L", "C_m", "a", "b", "tau_w", "I_e", "V_peak",
  "V_reset", "t_ref", "refractory_step", "den_delay"};

struct ModelShape {
  int n_port_var;
  const char *port_var[2];
  int n_port_par;
  const char *port_par[4];
  int input_var;       // index into port vars receiving spike input
  int weight_par;      // index into port params used as input weight (-1 = 1.0)
};

static ModelShape shape_of(Model m) {
  switch (m) {
  case AEIF_COND_BETA: return {2, {"g", "g1"}, 4, {"E_rev", "tau_rise", "tau_decay", "g0"}, 1, 3};
  case AEIF_COND_ALPHA: return {2, {"g", "g1"}, 3, {"E_rev", "tau_syn", "g0", nullptr}, 1, 2};
  case AEIF_PSC_EXP: return {1, {"I_syn", nullptr}, 1, {"tau_syn", nullptr, nullptr, nullptr}, 0, -1};
  case AEIF_PSC_ALPHA: return {2, {"I_syn", "I1_syn"}, 2, {"tau_syn", "I0", nullptr, nullptr}, 1, 1};
  default: return {0, {nullptr, nullptr}, 0, {nullptr, nullptr, nullptr, nullptr}, -1, -1};
  }
}

enum { I_I_syn_ex = 0, I_I_syn_in, I_V_m_rel, I_refractory_step, I_NVAR };
static const char *iaf_var_name[I_NVAR] = {"I_syn_ex", "I_syn_in", "V_m_rel", "refractory_step"};
enum { I_tau_m = 0, I_C_m, I_E_L, I_I_e, I_Theta_rel, I_V_reset_rel, I_tau_ex, I_tau_in,
       I_t_ref, I_den_delay, I_P20, I_P11ex, I_P11in, I_P21ex, I_P21in, I_P22, I_NPAR };
static const char *iaf_par_name[I_NPAR] = {
  "tau_m", "C_m", "E_L", "I_e", "Theta_rel", "V_reset_rel", "tau_ex", "tau_in",
  "t_ref", "den_delay", "P20", "P11ex", "P11in", "P21ex", "P21in", "P22"};

enum { PG_rate = 0, PG_origin, PG_start, PG_stop, PG_NPAR };
static const char *pg_par_name[PG_NPAR] = {"rate", "origin", "start", "stop"};

struct Group {
  Model model;
  int i0 = 0, n = 0, nport = 0;
  int lo = 0, hi = -1;                      // neurons simulated by this process (hi < 0: all)
  // aeif: scalar vars V_m,w ; port vars ; scalar params ; port params
  // iaf : vars (4) ; params (16)
  // poiss_gen: params (4)
  std::vector<std::vector<double>> var;     // [var][neuron] (port vars: [nscal + port*npv + v])
  std::vector<std::vector<double>> par;     // [param][neuron]
  float h_min_rel = 1.0e-3f, h0_rel = 1.0e-2f;
  std::vector<double> x;                    // aeif integration time
  std::vector<double> h;                    // aeif step size
  // spike generator
  std::vector<std::vector<int>> sg_tidx;
  std::vector<std::vector<float>> sg_height;
  std::vector<std::vector<float>> sg_times, sg_heights_set;
  std::vector<int> sg_next;
  // input accumulator [port][neuron]
  std::vector<double> acc;
  // recording
  bool spike_count_on = false;
  std::vector<int> spike_count;
  int max_rec = 0;
  std::vector<std::vector<float>> rec_times;
};

// ---------------------------------------------------------------------------
// Learned RK5 step-size proposal (no counterpart in the reference).  A CPU
// statement of the engine's network: features of a step, the 10-32-32-1 MLP with
// BF16-valued weights and FP32 accumulation (float fused multiply-adds in the
// kernel's order, so the result is bit-identical), and its exact FP64 gradient.
// Flat parameter vector: mu[10] inv_sigma[10] W1[32][10] b1[32] W2[32][32] b2[32]
// W3[32] b3 label_mu label_sigma safety floor (1465 floats); trainable block W1..b3.
// In the RK5 loop the proposal is raised to at least floor * (the controller's h).
// ---------------------------------------------------------------------------
namespace sm {
constexpr int NF = 10, NH = 32;
constexpr float XCLAMP = 8.0f;   // normalised inputs are clamped to [-8, 8]
constexpr int MU = 0, ISIG = MU + NF, W1 = ISIG + NF, B1 = W1 + NH * NF, W2 = B1 + NH, B2 = W2 + NH * NH,
              W3 = B2 + NH, B3 = W3 + NH, LMU = B3 + 1, LSIG = LMU + 1, SAFETY = LSIG + 1, FLOOR = SAFETY + 1,
              NPAR = FLOOR + 1;
constexpr int NTRAIN = B3 + 1 - W1;
constexpr int LOG_W = NF + 2;
}  // namespace sm

static float slog_f(float x) {   // sign(x) log(1 + |x|)
  const float l = log_m(1.0f + std::fabs(x));
  return (x < 0.0f) ? -l : l;
}

static float mlp_out_f(const float *M, const float *f) {
  using namespace sm;
  float xn[NF];
  for (int k = 0; k < NF; k++) {
    const float v = (f[k] - M[MU + k]) * M[ISIG + k];
    xn[k] = std::fmin(std::fmax(v, -XCLAMP), XCLAMP);
  }
  float a1[NH];
  for (int j = 0; j < NH; j++) {
    float z = M[B1 + j];
    for (int k = 0; k < NF; k++) z = std::fma(M[W1 + j * NF + k], xn[k], z);
    a1[j] = (z > 0.0f) ? z : 0.0f;
  }
  float out = M[B3];
  for (int j = 0; j < NH; j++) {
    float z = M[B2 + j];
    for (int k = 0; k < NH; k++) z = std::fma(M[W2 + j * NH + k], a1[k], z);
    z = (z > 0.0f) ? z : 0.0f;
    out = std::fma(M[W3 + j], z, out);
  }
  return out;
}

static float mlp_propose_f(const float *M, const float *f) {
  using namespace sm;
  return M[SAFETY] * exp_m(std::fma(mlp_out_f(M, f), M[LSIG], M[LMU]));
}

// Mean squared error over n samples of the normalised target (target - label_mu) /
// label_sigma, and its gradient with respect to the trainable block, in FP64.
static double mlp_grad_d(const float *M, const float *feat, const float *target, int n, double *grad) {
  using namespace sm;
  for (int o = 0; o < NTRAIN; o++) grad[o] = 0.0;
  double loss = 0.0;
  for (int s = 0; s < n; s++) {
    double xn[NF], z1[NH], a1[NH], z2[NH], a2[NH];
    for (int k = 0; k < NF; k++) {
      // the clamp is applied in FP32, as in the engine
      const float v = (feat[s * NF + k] - M[MU + k]) * M[ISIG + k];
      xn[k] = (double)std::fmin(std::fmax(v, -XCLAMP), XCLAMP);
    }
    for (int j = 0; j < NH; j++) {
      double z = M[B1 + j];
      for (int k = 0; k < NF; k++) z += (double)M[W1 + j * NF + k] * xn[k];
      z1[j] = z;
      a1[j] = z > 0 ? z : 0;
    }
    double out = M[B3];
    for (int j = 0; j < NH; j++) {
      double z = M[B2 + j];
      for (int k = 0; k < NH; k++) z += (double)M[W2 + j * NH + k] * a1[k];
      z2[j] = z;
      a2[j] = z > 0 ? z : 0;
      out += (double)M[W3 + j] * a2[j];
    }
    const double tn = ((double)target[s] - M[LMU]) / (double)M[LSIG];
    const double r = out - tn;
    loss += r * r;
    const double d = 2.0 * r / n;
    double d2[NH], d1[NH];
    for (int j = 0; j < NH; j++) d2[j] = z2[j] > 0 ? d * M[W3 + j] : 0.0;
    for (int k = 0; k < NH; k++) {
      double g = 0;
      for (int j = 0; j < NH; j++) g += (double)M[W2 + j * NH + k] * d2[j];
      d1[k] = z1[k] > 0 ? g : 0.0;
    }
    for (int j = 0; j < NH; j++) {
      for (int k = 0; k < NF; k++) grad[W1 - W1 + j * NF + k] += d1[j] * xn[k];
      grad[B1 - W1 + j] += d1[j];
      for (int k = 0; k < NH; k++) grad[W2 - W1 + j * NH + k] += d2[j] * a1[k];
      grad[B2 - W1 + j] += d2[j];
      grad[W3 - W1 + j] += d * a2[j];
    }
    grad[B3 - W1] += d;
  }
  return loss / n;
}

// Nearest BF16 value of a float, ties to even (finite inputs), as a float.
static float bf16r(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// mlp_grad_d with the operands of the engine's tensor-core training kernel rounded to BF16
// where they enter a product: the normalised inputs, the layer-1 activations (FP32 first),
// the layer-2 errors and the output error for the products, the layer-1 errors and the
// layer-2 activations for the weight gradients; everything else in FP64.
static double mlp_grad_bf16_d(const float *M, const float *feat, const float *target, int n, double *grad) {
  using namespace sm;
  for (int o = 0; o < NTRAIN; o++) grad[o] = 0.0;
  double loss = 0.0;
  for (int s = 0; s < n; s++) {
    double xb[NF], z1[NH], a1b[NH], z2[NH], a2[NH];
    for (int k = 0; k < NF; k++) {
      const float v = (feat[s * NF + k] - M[MU + k]) * M[ISIG + k];
      xb[k] = (double)bf16r(std::fmin(std::fmax(v, -XCLAMP), XCLAMP));
    }
    for (int j = 0; j < NH; j++) {
      double z = 0.0;
      for (int k = 0; k < NF; k++) z += (double)M[W1 + j * NF + k] * xb[k];
      z1[j] = z + M[B1 + j];
      a1b[j] = z1[j] > 0 ? (double)bf16r((float)z1[j]) : 0.0;
    }
    double out = M[B3];
    for (int j = 0; j < NH; j++) {
      double z = 0.0;
      for (int k = 0; k < NH; k++) z += (double)M[W2 + j * NH + k] * a1b[k];
      z2[j] = z + M[B2 + j];
      a2[j] = z2[j] > 0 ? z2[j] : 0;
      out += (double)M[W3 + j] * a2[j];
    }
    const double tn = ((double)target[s] - M[LMU]) / (double)M[LSIG];
    const double r = out - tn;
    loss += r * r;
    const double d = 2.0 * r / n;
    const double db = (double)bf16r((float)d);
    double d2b[NH], d1b[NH];
    for (int j = 0; j < NH; j++) d2b[j] = z2[j] > 0 ? (double)bf16r((float)(d * M[W3 + j])) : 0.0;
    for (int k = 0; k < NH; k++) {
      double g = 0;
      for (int j = 0; j < NH; j++) g += (double)M[W2 + j * NH + k] * d2b[j];
      d1b[k] = z1[k] > 0 ? (double)bf16r((float)g) : 0.0;
    }
    for (int j = 0; j < NH; j++) {
      for (int k = 0; k < NF; k++) grad[W1 - W1 + j * NF + k] += d1b[j] * xb[k];
      grad[B1 - W1 + j] += d1b[j];
      for (int k = 0; k < NH; k++) grad[W2 - W1 + j * NH + k] += d2b[j] * a1b[k];
      grad[B2 - W1 + j] += d2b[j];
      grad[W3 - W1 + j] += db * (double)bf16r((float)a2[j]);
    }
    grad[B3 - W1] += db;
  }
  return loss / n;
}

struct Queued { int age; int cursor; float height; };

// syn: synapse group (0: static, k: syn_groups[k-1]); stamp: low 16 bits of the time index
// of the last spike that arrived through the edge (plastic edges), 0x8000 initially
// (src/rev_spike.cu:150-155)
struct Edge { int tgt; unsigned char port; float w; unsigned char syn = 0; unsigned short stamp = 0x8000; };

// Synapse models (src/syn_model.h, src/stdp.h:70-94, src/test_syn_model.h)
enum SynType { SYN_TEST = 0, SYN_STDP = 1 };
struct SynGroupDef { int type; std::vector<float> par; };
static const char *const kStdpPar[] = {"tau_plus", "tau_minus", "lambda", "alpha", "mu_plus", "mu_minus", "Wmax"};
static const char *const kTestPar[] = {"fact", "offset"};
constexpr int kMaxSynDt = 16384;                 // MAX_SYN_DT, src/syn_model.h:33
constexpr long long kLastSpikeGuard = 0x70000000LL;   // src/spike_buffer.cu:42

// SynapseUpdate (src/syn_model.cu:43-56): STDPUpdate (src/stdp.cu:36-64) in FP64, or the
// test model's linear rule (src/test_syn_model.cu:35-40).
static float synapse_update(const SynGroupDef &g, float w, float Dt) {
  if (g.type == SYN_TEST) {
    const float fact = g.par[0], offset = g.par[1];
    return w + std::fma(fact, Dt, offset);
  }
  const double tau_plus = g.par[0], tau_minus = g.par[1], lambda = g.par[2], alpha = g.par[3];
  const double mu_plus = g.par[4], mu_minus = g.par[5], Wmax = g.par[6];
  const double wd = w;
  double w1;
  if (Dt >= 0) {
    const double fact = lambda * std::exp(-(double)Dt / tau_plus);
    w1 = wd + fact * Wmax * std::pow(1.0 - wd / Wmax, mu_plus);
  } else {
    const double fact = -alpha * lambda * std::exp((double)Dt / tau_minus);
    w1 = wd + fact * Wmax * std::pow(wd / Wmax, mu_minus);
  }
  w1 = w1 > 0.0 ? w1 : 0.0;
  w1 = w1 < Wmax ? w1 : Wmax;
  return (float)w1;
}
struct DelayGroup { int delay; std::vector<Edge> tg; };

struct Rec { int node; std::string var; int port; };

struct Net {
  bool fp64 = false;
  float dt = 0.1f;
  unsigned long long seed = 54321ULL;
  unsigned long long kernel_seed = 54321ULL + 12345ULL;
  curandGenerator_t gen = nullptr;
  int max_spike_buffer = 20;
  std::vector<Group> groups;
  std::vector<int> node_group;
  std::vector<std::vector<DelayGroup>> conn;     // per source, delays ascending
  std::vector<SynGroupDef> syn_groups;
  bool any_plastic = false;
  std::vector<long long> last_rev;                // per node: time index of the last spike
                                                  // to reach the node's synapses
  std::vector<int> den_steps;                     // per node: dendritic delay in steps
  std::map<long long, std::vector<int>> rev_pending;   // time index -> nodes whose spike arrives
  std::vector<std::vector<Edge *>> rev_in;        // per node: incoming plastic edges
  // simulation state
  bool calibrated = false;
  bool first_sim = true;
  double neural_time = 0.0, neur_t0 = 0.0;
  long long it = 0, Nt = 0;
  std::vector<std::vector<Queued>> queue;         // per source, most recent first
  // direct (poiss_gen) edges in canonical order
  // Poisson stream of an edge: (stream, out-edge index of its generator in connection
  // order); stream = the generator's index among all poiss_gen nodes unless set
  struct Direct { int gen; int tgt; unsigned char port; float w; float delay; int group; uint64_t key; };
  std::vector<Direct> direct;
  std::map<int, uint32_t> pg_stream;              // poiss_gen node -> stream (set explicitly)
  // partitioned network: this process simulates its share of every group; after the update
  // phase of each step xch_fn exchanges the step's spikes (orc_step_spikes / orc_inject_spikes)
  int part_rank = 0, part_world = 1;
  struct StepSpike { int node; float height; };
  std::vector<StepSpike> step_spikes;
  bool injecting = false;
  int (*xch_fn)(void *) = nullptr;
  void *xch_user = nullptr;
  long long cur_tidx = 0;
  std::vector<Rec> recs;
  std::vector<std::vector<float>> rec_rows;
  long long n_derivs = 0;
  long long n_rk5_steps = 0, n_rk5_trials = 0;
  // learned step size: 0 plain, 1 log tuples, 2 network proposal, 3 best possible proposal
  // (every step starts from the largest step that passes the unchanged error test, found
  // by bisection; an analysis bound, FP32 mode only)
  int learn_mode = 0;
  std::vector<float> model;
  std::vector<float> steplog;
  long long log_cap = 0, log_offered = 0;
  long long n_spikes_total = 0;
  long long n_events = 0;    // synaptic events delivered (edges traversed)
  std::string err;

  Net() { reseed(54321ULL); }
  ~Net() { if (gen) curandDestroyGenerator(gen); }

  void reseed(unsigned long long s) {
    seed = s;
    kernel_seed = s + 12345ULL;
    if (gen) curandDestroyGenerator(gen);
    if (curandCreateGeneratorHost(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS)
      throw std::runtime_error("curandCreateGeneratorHost failed");
    curandSetPseudoRandomGeneratorSeed(gen, s);
  }

  std::vector<unsigned int> random_int(size_t n) {
    std::vector<unsigned int> v(n);
    if (n && curandGenerate(gen, v.data(), n) != CURAND_STATUS_SUCCESS)
      throw std::runtime_error("curandGenerate failed");
    return v;
  }
  std::vector<float> random_normal(size_t n, float mean, float sd) {
    size_t n1 = (n % 2 == 0) ? n : n + 1;
    std::vector<float> v(n1);
    if (n1 && curandGenerateNormal(gen, v.data(), n1, mean, sd) != CURAND_STATUS_SUCCESS)
      throw std::runtime_error("curandGenerateNormal failed");
    v.resize(n);
    return v;
  }
  std::vector<float> random_uniform(size_t n) {
    std::vector<float> v(n);
    if (n && curandGenerateUniform(gen, v.data(), n) != CURAND_STATUS_SUCCESS)
      throw std::runtime_error("curandGenerateUniform failed");
    return v;
  }
  // src/nestgpu.cu:1150-1188
  std::vector<float> random_normal_clipped(size_t n, float mean, float sd, float vmin,
                                           float vmax, float vstep) {
    const float epsi = 1.0e-6f;
    n = (n / 4 + 1) * 4;
    int n_extra = (int)(n / 10);
    n_extra = (n_extra / 4 + 1) * 4;
    if (n_extra < 1024) n_extra = 1024;
    int i_extra = 0;
    std::vector<float> arr = random_normal(n, mean, sd);
    std::vector<float> extra;
    for (size_t i = 0; i < n; i++) {
      while (arr[i] < vmin || arr[i] > vmax) {
        if (i_extra == 0) extra = random_normal(n_extra, mean, sd);
        arr[i] = extra[i_extra];
        i_extra++;
        if (i_extra == n_extra) i_extra = 0;
      }
    }
    if (vstep > sd * epsi) {
      for (size_t i = 0; i < n; i++)
        arr[i] = vmin + vstep * std::round((arr[i] - vmin) / vstep);
    }
    return arr;
  }

  Group &group_of(int node) {
    if (node < 0 || node >= (int)node_group.size()) throw std::runtime_error("node out of range");
    return groups[node_group[node]];
  }

  int create(const std::string &name, int n, int nport) {
    if (calibrated) throw std::runtime_error("Nodes cannot be created after calibration");
    if (n <= 0) throw std::runtime_error("Number of nodes must be greater than zero.");
    int m = -1;
    for (int i = 0; i < N_MODEL; i++) if (name == model_name[i]) m = i;
    if (m < 0) throw std::runtime_error("Unknown neuron model name");
    Group g;
    g.model = (Model)m;
    g.i0 = (int)node_group.size();
    g.n = n;
    if (is_aeif(g.model)) {
      g.nport = nport;
      ModelShape s = shape_of(g.model);
      g.var.assign(2 + s.n_port_var * nport, std::vector<double>(n, 0.0));
      g.par.assign(A_NSCAL + s.n_port_par * nport, std::vector<double>(n, 0.0));
      double d[A_NSCAL] = {-50.4, 2.0, 30.0, -70.6, 281.0, 4.0, 80.5, 144.0, 0.0, 0.0, -60.0, 0.0, 0.0, 0.0};
      for (int j = 0; j < A_NSCAL; j++) std::fill(g.par[j].begin(), g.par[j].end(), (double)(float)d[j]);
      std::fill(g.var[0].begin(), g.var[0].end(), (double)(float)-70.6);
      for (int p = 0; p < nport; p++) {
        auto P = [&](int k) -> std::vector<double> & { return g.par[A_NSCAL + s.n_port_par * p + k]; };
        switch (g.model) {
        case AEIF_COND_BETA:
          std::fill(P(0).begin(), P(0).end(), 0.0);
          std::fill(P(1).begin(), P(1).end(), 2.0);
          std::fill(P(2).begin(), P(2).end(), 20.0);
          break;
        case AEIF_COND_ALPHA:
          std::fill(P(0).begin(), P(0).end(), 0.0);
          std::fill(P(1).begin(), P(1).end(), 2.0);
          break;
        case AEIF_PSC_EXP:
        case AEIF_PSC_ALPHA:
          std::fill(P(0).begin(), P(0).end(), (double)0.2f);
          break;
        default: break;
        }
      }
      g.x.assign(n, 0.0);
      g.h.assign(n, (double)(g.h0_rel * 0.1f));
    } else if (g.model == IAF_PSC_EXP) {
      g.nport = 2;
      g.var.assign(I_NVAR, std::vector<double>(n, 0.0));
      g.par.assign(I_NPAR, std::vector<double>(n, 0.0));
      double d[10] = {10.0, 250.0, -70.0, 0.0, 15.0, 0.0, 2.0, 2.0, 2.0, 0.0};
      for (int j = 0; j < 10; j++) std::fill(g.par[j].begin(), g.par[j].end(), d[j]);
    } else if (g.model == SPIKE_GEN) {
      g.nport = 0;
      g.sg_tidx.assign(n, {});
      g.sg_height.assign(n, {});
      g.sg_times.assign(n, {});
      g.sg_heights_set.assign(n, {});
      g.sg_next.assign(n, 0);
    } else if (g.model == POISS_GEN) {
      g.nport = 0;
      g.par.assign(PG_NPAR, std::vector<double>(n, 0.0));
      std::fill(g.par[PG_stop].begin(), g.par[PG_stop].end(), (double)1.0e30f);
    } else if (g.model == PARROT) {
      g.nport = 2;
      g.var.assign(PR_NVAR, std::vector<double>(n, 0.0));
      g.par.assign(PR_NPAR, std::vector<double>(n, 0.0));
    } else if (g.model == SPIKE_DET) {
      g.nport = 1;
      g.var.assign(SD_NVAR, std::vector<double>(n, 0.0));
      g.par.assign(SD_NPAR, std::vector<double>(n, 1.0));
    }
    g.acc.assign((size_t)g.nport * n, 0.0);
    groups.push_back(g);
    node_group.insert(node_group.end(), n, (int)groups.size() - 1);
    conn.resize(node_group.size());
    return g.i0;
  }

  // Locate a named quantity. kind: 0 scal var, 1 port var, 2 scal param, 3 port param,
  // 4 group param, 5 array param (spike gen).  Returns index or -1.
  int locate(Group &g, const std::string &name, int &kind) {
    if (is_aeif(g.model)) {
      ModelShape s = shape_of(g.model);
      if (name == "V_m") { kind = 0; return 0; }
      if (name == "w") { kind = 0; return 1; }
      for (int k = 0; k < s.n_port_var; k++) if (name == s.port_var[k]) { kind = 1; return k; }
      for (int k = 0; k < A_NSCAL; k++) if (name == aeif_scal_name[k]) { kind = 2; return k; }
      for (int k = 0; k < s.n_port_par; k++) if (name == s.port_par[k]) { kind = 3; return k; }
      if (name == "h_min_rel") { kind = 4; return 0; }
      if (name == "h0_rel") { kind = 4; return 1; }
    } else if (g.model == IAF_PSC_EXP) {
      for (int k = 0; k < I_NVAR; k++) if (name == iaf_var_name[k]) { kind = 0; return k; }
      for (int k = 0; k < I_NPAR; k++) if (name == iaf_par_name[k]) { kind = 2; return k; }
    } else if (g.model == POISS_GEN) {
      for (int k = 0; k < PG_NPAR; k++) if (name == pg_par_name[k]) { kind = 2; return k; }
    } else if (g.model == PARROT) {
      for (int k = 0; k < PR_NVAR; k++) if (name == parrot_var_name[k]) { kind = 0; return k; }
      for (int k = 0; k < PR_NPAR; k++) if (name == parrot_par_name[k]) { kind = 2; return k; }
    } else if (g.model == SPIKE_DET) {
      for (int k = 0; k < SD_NVAR; k++) if (name == sdet_var_name[k]) { kind = 0; return k; }
      for (int k = 0; k < SD_NPAR; k++) if (name == sdet_par_name[k]) { kind = 2; return k; }
    } else if (g.model == SPIKE_GEN) {
      if (name == "spike_times") { kind = 5; return 0; }
      if (name == "spike_heights") { kind = 5; return 1; }
    }
    return -1;
  }

  std::vector<double> &slot(Group &g, int kind, int idx, int port) {
    if (kind == 0) return g.var[idx];
    if (kind == 2) return g.par[idx];
    ModelShape s = shape_of(g.model);
    if (port < 0 || port >= g.nport) throw std::runtime_error("port out of range");
    if (kind == 1) return g.var[2 + s.n_port_var * port + idx];
    return g.par[A_NSCAL + s.n_port_par * port + idx];
  }

  void set_value(int node, const std::string &name, int port, float val) {
    Group &g = group_of(node);
    int kind;
    int idx = locate(g, name, kind);
    if (idx < 0) throw std::runtime_error("Unrecognized variable or parameter " + name);
    int i = node - g.i0;
    if (kind == 4) {
      if (idx == 0) g.h_min_rel = val; else g.h0_rel = val;
      return;
    }
    if (kind == 5) throw std::runtime_error("array parameter needs an array");
    slot(g, kind, idx, port)[i] = (double)val;
  }

  float get_value(int node, const std::string &name, int port) {
    Group &g = group_of(node);
    int kind;
    int idx = locate(g, name, kind);
    int i = node - g.i0;
    if (name == "spike_count") {
      if (!g.spike_count_on) throw std::runtime_error("spike count not active");
      return (float)g.spike_count[i];
    }
    if (idx < 0) throw std::runtime_error("Unrecognized variable or parameter " + name);
    if (kind == 4) return idx == 0 ? g.h_min_rel : g.h0_rel;
    if (kind == 5) throw std::runtime_error("array parameter");
    return (float)slot(g, kind, idx, port)[i];
  }

  void set_spike_times(int node, int n, const float *t, const float *h) {
    Group &g = group_of(node);
    if (g.model != SPIKE_GEN) throw std::runtime_error("not a spike generator");
    int i = node - g.i0;
    g.sg_times[i].assign(t, t + n);
    if (h) g.sg_heights_set[i].assign(h, h + n); else g.sg_heights_set[i].clear();
  }

  // src/connect.cu:38-74
  void connect1(int src, int tgt, int port, float w, float delay, int syn = 0) {
    if (delay < dt) throw std::runtime_error("Delay must be >= time resolution");
    if (syn < 0 || syn > (int)syn_groups.size()) throw std::runtime_error("Unrecognized synapse group");
    if (syn > 0) any_plastic = true;
    connect_step(src, tgt, port, w, (int)std::round(delay / dt) - 1, syn);
  }

  // insertion into the source's delay group d_int (src/connect.cu:38-74: groups ascending
  // by delay, targets in insertion order)
  void connect_step(int src, int tgt, int port, float w, int d_int, int syn = 0) {
    std::vector<DelayGroup> &c = conn[src];
    size_t id = 0;
    while (id < c.size() && d_int > c[id].delay) id++;
    if (id == c.size() || d_int != c[id].delay) {
      DelayGroup ng;
      ng.delay = d_int;
      Edge e{tgt, (unsigned char)port, w};
      e.syn = (unsigned char)syn;
      ng.tg.push_back(e);
      c.insert(c.begin() + id, ng);
    } else {
      Edge e{tgt, (unsigned char)port, w};
      e.syn = (unsigned char)syn;
      c[id].tg.push_back(e);
    }
  }

  // The engine's generated fixed in-degree block (ConnectFixedIndegreeGPU; no reference
  // counterpart: it stands in for src/connect_rules.h:203-269 in the large benchmark
  // networks, with sources drawn per target and with replacement).  Edge kk of the block's
  // t-th target: one Philox4x32-10 block keyed by the seed with counter (t, kk, 0,
  // 0x9E3779B9); source = src0 + floor(x * ns / 2^32), delay step = dlo + floor(y * (dhi -
  // dlo + 1) / 2^32) with dlo/dhi = round(delay_min/max / dt) - 1.
  void connect_generated(int src0, int ns, int tgt0, int nt, int k, int port, float w, float dmin_ms,
                         float dmax_ms, uint64_t seed) {
    if (calibrated) throw std::runtime_error("Connections cannot be created after calibration");
    if (ns <= 0 || nt <= 0 || k <= 0) throw std::runtime_error("empty connection block");
    if (dmin_ms < dt || dmax_ms < dmin_ms) throw std::runtime_error("Delay must be >= time resolution");
    const int dlo = (int)std::round(dmin_ms / dt) - 1;
    const int dhi = (int)std::round(dmax_ms / dt) - 1;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int t = 0; t < nt; t++)
      for (int kk = 0; kk < k; kk++) {
        U4 r = philox({(uint32_t)t, (uint32_t)kk, 0u, 0x9E3779B9u}, k0, k1);
        const int s = src0 + (int)(((uint64_t)r.x * (uint32_t)ns) >> 32);
        const int d = dlo + (int)(((uint64_t)r.y * (uint32_t)(dhi - dlo + 1)) >> 32);
        connect_step(s, tgt0 + t, port, w, d, 0);
      }
  }

  // src/connect_rules.h:161-338 (one host thread: THREAD_MAXNUM == 1)
  void connect_rule(int rule, const int *src_arr, int src0, int ns, const int *tgt_arr, int tgt0,
                    int nt, int degree, int port, int syn, float weight, float delay,
                    const float *warr, const float *darr) {
    if (calibrated) throw std::runtime_error("Connections cannot be created after calibration");
    auto S = [&](int i) { return src_arr ? src_arr[i] : src0 + i; };
    auto T = [&](int i) { return tgt_arr ? tgt_arr[i] : tgt0 + i; };
    auto one = [&](int is, int it_, size_t ia) {
      float w = warr ? warr[ia] : weight;
      float d = darr ? darr[ia] : delay;
      connect1(S(is), T(it_), port, w, d, syn);
    };
    enum { ONE_TO_ONE = 0, ALL_TO_ALL, FIXED_TOTAL_NUMBER, FIXED_INDEGREE, FIXED_OUTDEGREE };
    const int thresh = 5;
    switch (rule) {
    case ONE_TO_ONE:
      if (ns != nt) throw std::runtime_error("Number of source and target nodes must be equal for the one-to-one connection rule");
      for (int i = 0; i < ns; i++) one(i, i, (size_t)i);
      break;
    case ALL_TO_ALL:
      for (int itn = 0; itn < nt; itn++)
        for (int isn = 0; isn < ns; isn++) one(isn, itn, (size_t)itn * ns + isn);
      break;
    case FIXED_TOTAL_NUMBER: {
      std::vector<unsigned int> rnd = random_int(2 * (size_t)degree);
      for (int i = 0; i < degree; i++) one((int)(rnd[2 * i] % ns), (int)(rnd[2 * i + 1] % nt), (size_t)i);
      break;
    }
    case FIXED_INDEGREE:
    case FIXED_OUTDEGREE: {
      bool in = rule == FIXED_INDEGREE;
      int npool = in ? ns : nt;
      int nloop = in ? nt : ns;
      if (degree > npool)
        throw std::runtime_error(in ? "Indegree larger than number of source nodes"
                                    : "Outdegree larger than number of target nodes");
      size_t n_rnd = degree;
      if (npool >= thresh * degree) n_rnd *= 5;
      std::vector<unsigned int> rnd = random_int(n_rnd);
      for (int k = 0; k < nloop; k++) {
        std::vector<int> pick;
        if (npool < thresh * degree) {
          pick.resize(npool);
          std::iota(pick.begin(), pick.end(), 0);
          for (int i = 0; i < degree; i++) {
            int j = i + (int)(rnd[i] % (unsigned)(npool - i));
            if (j != i) std::swap(pick[i], pick[j]);
          }
        } else {
          std::vector<int> sorted;
          for (int i = 0; i < degree; i++) {
            int i1 = 0;
            std::vector<int>::iterator itr;
            int j;
            do {
              size_t ri = (size_t)i1 * degree + i;
              // the reference reads past its buffer after five collisions
              if (ri >= rnd.size()) throw std::runtime_error("fixed-degree draw exhausted its random buffer");
              j = (int)(rnd[ri] % (unsigned)npool);
              itr = std::lower_bound(sorted.begin(), sorted.end(), j);
              i1++;
            } while (itr != sorted.end() && *itr == j);
            sorted.insert(itr, j);
            pick.push_back(j);
          }
        }
        for (int i = 0; i < degree; i++) {
          if (in) one(pick[i], k, (size_t)k * degree + i);
          else one(k, pick[i], (size_t)k * degree + i);
        }
      }
      break;
    }
    default: throw std::runtime_error("Unknown connection rule");
    }
  }

  // -------------------------------------------------------------- calibrate
  static double propagator_32(double tau_syn, double tau, double C, double h) {
    const double P32_linear = 1.0 / (2.0 * C * tau * tau) * h * h * (tau_syn - tau) * std::exp(-h / tau);
    const double P32_singular = h / C * std::exp(-h / tau);
    const double P32 = -tau / (C * (1.0 - tau / tau_syn)) * std::exp(-h / tau_syn) *
                       std::expm1(h * (1.0 / tau_syn - 1.0 / tau));
    const double dev_P32 = std::fabs(P32 - P32_singular);
    if (tau == tau_syn || (std::fabs(tau - tau_syn) < 0.1 && dev_P32 > 2.0 * std::fabs(P32_linear)))
      return P32_singular;
    return P32;
  }

  void calibrate() {
    if (calibrated) throw std::runtime_error("Calibration can be made only once");
    calibrated = true;
    for (auto &g : groups) {
      if (part_world > 1) {
        g.lo = (int)((long long)g.n * part_rank / part_world);
        g.hi = (int)((long long)g.n * (part_rank + 1) / part_world);
      } else {
        g.lo = 0;
        g.hi = -1;
      }
    }
    neural_time = 0.0;
    queue.assign(node_group.size(), {});
    // direct edges: poiss_gen sources, source-major, delay groups ascending, insertion order
    direct.clear();
    uint32_t ordinal = 0;
    for (size_t gi = 0; gi < groups.size(); gi++) {
      Group &g = groups[gi];
      if (g.model != POISS_GEN) continue;
      for (int s = g.i0; s < g.i0 + g.n; s++, ordinal++) {
        auto it = pg_stream.find(s);
        const uint64_t stream = it != pg_stream.end() ? it->second : ordinal;
        uint32_t local = 0;
        for (auto &dg : conn[s])
          for (auto &e : dg.tg)
            direct.push_back({s - g.i0, e.tgt, e.port, e.w, dt * (float)(dg.delay + 1), (int)gi,
                              (stream << 32) | (uint64_t)(local++)});
      }
    }
    for (auto &g : groups) {
      if (is_aeif(g.model)) {
        ModelShape s = shape_of(g.model);
        for (int i = 0; i < g.n; i++) {
          g.par[A_refractory_step][i] = 0.0;
          for (int p = 0; p < g.nport; p++) {
            auto P = [&](int k) -> double & { return g.par[A_NSCAL + s.n_port_par * p + k][i]; };
            if (g.model == AEIF_COND_BETA) {
              float td = (float)P(2), tr = (float)P(1);
              float denom1 = td - tr;
              float denom2 = 0.0f;
              float g0;
              if (denom1 != 0.0f) {
                float t_p = td * tr * logf(td / tr) / denom1;
                denom2 = expf(-t_p / td) - expf(-t_p / tr);
              }
              if (denom2 == 0.0f) g0 = (float)(M_E / td);
              else g0 = (float)((1.0 / tr - 1.0 / td) / denom2);
              P(3) = g0;
            } else if (g.model == AEIF_COND_ALPHA) {
              P(2) = (float)(M_E / (float)P(1));
            } else if (g.model == AEIF_PSC_ALPHA) {
              P(1) = (float)(M_E / (float)P(0));
            }
          }
          if ((g.model == AEIF_PSC_EXP || g.model == AEIF_PSC_ALPHA) && g.par[A_Delta_T][i] <= 0.0)
            g.par[A_V_peak][i] = g.par[A_V_th][i];
          g.x[i] = 0.0;
          g.h[i] = (double)(g.h0_rel * dt);
        }
      } else if (g.model == IAF_PSC_EXP) {
        for (int i = 0; i < g.n; i++) {
          double h = dt;
          double tau_m = (float)g.par[I_tau_m][i], C_m = (float)g.par[I_C_m][i];
          double tau_ex = (float)g.par[I_tau_ex][i], tau_in = (float)g.par[I_tau_in][i];
          float P22 = (float)std::exp(-h / tau_m);
          g.par[I_P11ex][i] = (float)std::exp(-h / tau_ex);
          g.par[I_P11in][i] = (float)std::exp(-h / tau_in);
          g.par[I_P22][i] = P22;
          g.par[I_P21ex][i] = (float)propagator_32(tau_ex, tau_m, C_m, h);
          g.par[I_P21in][i] = (float)propagator_32(tau_in, tau_m, C_m, h);
          g.par[I_P20][i] = (float)(tau_m / C_m * (1.0 - (double)P22));
        }
      } else if (g.model == SPIKE_GEN) {
        for (int i = 0; i < g.n; i++) {
          int ns = (int)g.sg_times[i].size();
          g.sg_tidx[i].clear();
          g.sg_height[i].clear();
          if (ns == 0) continue;
          std::vector<float> hh = g.sg_heights_set[i];
          if (hh.empty()) hh.assign(ns, 1.0f);
          else if ((int)hh.size() != ns)
            throw std::runtime_error("spike time array and spike height array must have the same size in spike generator");
          for (int k = 0; k < ns; k++) {
            int ti = (int)std::round((g.sg_times[i][k] - 0.0f) / dt);
            if (k > 0 && ti <= g.sg_tidx[i][k - 1])
              throw std::runtime_error("Spike times must be ordered, and the difference between\nconsecutive spikes must be >= the time resolution");
            g.sg_tidx[i].push_back(ti);
            g.sg_height[i].push_back(hh[k]);
          }
          g.sg_next[i] = 0;
        }
      }
    }
    // check ports of recurrent connections
    for (size_t s = 0; s < conn.size(); s++)
      for (auto &dg : conn[s])
        for (auto &e : dg.tg) {
          Group &tg = groups[node_group[e.tgt]];
          if (e.port >= tg.nport) throw std::runtime_error("receptor port out of range for target node");
        }
    // plastic edges: per target the incoming ones (src/spike_buffer.cu:430-520), and the
    // last spike time index of every node (src/spike_buffer.cu:319-328)
    last_rev.assign(node_group.size(), kLastSpikeGuard);
    rev_in.assign(node_group.size(), {});
    // dendritic delay in steps, round(den_delay / dt) in float (src/spike_buffer.cu:175-177)
    den_steps.assign(node_group.size(), 0);
    for (auto &g : groups) {
      const std::vector<double> *dd = nullptr;
      if (is_aeif(g.model)) dd = &g.par[A_den_delay];
      else if (g.model == IAF_PSC_EXP) dd = &g.par[I_den_delay];
      else if (g.model == PARROT) dd = &g.par[PR_den_delay];
      if (dd)
        for (int i = 0; i < g.n; i++) den_steps[g.i0 + i] = (int)std::round((float)(*dd)[i] / dt);
    }
    if (any_plastic)
      for (size_t s = 0; s < conn.size(); s++) {
        if (groups[node_group[s]].model == POISS_GEN)
          for (auto &dg : conn[s])
            for (auto &e : dg.tg)
              if (e.syn) throw std::runtime_error("poiss_gen connections cannot be plastic");
        for (auto &dg : conn[s])
          for (auto &e : dg.tg)
            if (e.syn) rev_in[e.tgt].push_back(&e);
      }
  }

  // ---------------------------------------------------------------- stepping
  template <class R> struct C5 {
    R c2, c3, c4, c5, c6, a21, a31, a32, a41, a42, a43, a51, a52, a53, a54, a61, a62, a63, a64,
        a65, a71, a73, a74, a76, e1, e3, e4, e5, e6, eps, coeff, exp_inc, exp_dec, err_min, scal_min;
    C5() {
      c2 = (R)0.2; c3 = (R)0.3; c4 = (R)0.6; c5 = (R)1.0; c6 = (R)0.875;
      a21 = (R)0.2; a31 = (R)(3.0 / 40.0); a32 = (R)(9.0 / 40.0);
      a41 = (R)0.3; a42 = (R)-0.9; a43 = (R)1.2;
      a51 = (R)(-11.0 / 54.0); a52 = (R)2.5; a53 = (R)(-70.0 / 27.0); a54 = (R)(35.0 / 27.0);
      a61 = (R)(1631.0 / 55296.0); a62 = (R)(175.0 / 512.0); a63 = (R)(575.0 / 13824.0);
      a64 = (R)(44275.0 / 110592.0); a65 = (R)(253.0 / 4096.0);
      a71 = (R)(37.0 / 378.0); a73 = (R)(250.0 / 621.0); a74 = (R)(125.0 / 594.0); a76 = (R)(512.0 / 1771.0);
      e1 = (R)(37.0 / 378.0 - 2825.0 / 27648.0); e3 = (R)(250.0 / 621.0 - 18575.0 / 48384.0);
      e4 = (R)(125.0 / 594.0 - 13525.0 / 55296.0); e5 = (R)(-277.00 / 14336.0);
      e6 = (R)(512.0 / 1771.0 - 0.25);
      eps = (R)1.0e-6; coeff = (R)0.9; exp_inc = (R)-0.2; exp_dec = (R)-0.25;
      err_min = (R)1.889568e-4; scal_min = (R)1.0e-1;
    }
  };

  // Per-neuron, per-model RHS.  y layout: V_m, w, then port vars (port-major).
  template <class R> struct Par {
    R V_th, Delta_T, inv_Delta_T, g_L, E_L, C_m, inv_C_m, a, b, tau_w, inv_tau_w, I_e, V_peak,
        V_reset, t_ref;
    R E_rev[32], t1[32], inv_t1[32], t2[32], inv_t2[32];
  };

  static inline float fmaR(float a, float b, float c) { return std::fmaf(a, b, c); }
  static inline double fmaR(double a, double b, double c) { return std::fma(a, b, c); }

  template <class R>
  void derivs(Model m, int P, const R *y, R *dy, const Par<R> &q, R refr) {
    R V = (refr > (R)0) ? q.V_reset : ((y[0] < q.V_peak) ? y[0] : q.V_peak);
    const R w = y[1];
    R I = (R)0;
    bool cond = (m == AEIF_COND_BETA || m == AEIF_COND_ALPHA);
    int npv = (m == AEIF_PSC_EXP) ? 1 : 2;
    if (fp64) {
      if (cond) {
        for (int i = 0; i < P; i++) I += y[2 + 2 * i] * (q.E_rev[i] - V);
      } else {
        for (int i = 0; i < P; i++) I += y[2 + npv * i];
      }
      R Vs;
      if (!cond && q.Delta_T == (R)0) Vs = (R)0;
      else Vs = q.Delta_T * (R)std::exp((double)((V - q.V_th) / q.Delta_T));
      dy[0] = (refr > (R)0) ? (R)0 : (-q.g_L * (V - q.E_L - Vs) + I - w + q.I_e) / q.C_m;
      dy[1] = (q.a * (V - q.E_L) - w) / q.tau_w;
      for (int i = 0; i < P; i++) {
        if (m == AEIF_COND_BETA) {
          dy[3 + 2 * i] = -y[3 + 2 * i] / q.t1[i];
          dy[2 + 2 * i] = y[3 + 2 * i] - y[2 + 2 * i] / q.t2[i];
        } else if (m == AEIF_COND_ALPHA || m == AEIF_PSC_ALPHA) {
          dy[3 + 2 * i] = -y[3 + 2 * i] / q.t1[i];
          dy[2 + 2 * i] = y[3 + 2 * i] - y[2 + 2 * i] / q.t1[i];
        } else {
          dy[2 + i] = -y[2 + i] / q.t1[i];
        }
      }
      return;
    }
    // FP32 mirror of the CUDA kernel arithmetic
    if (cond) {
      for (int i = 0; i < P; i++) I = fmaR(y[2 + 2 * i], q.E_rev[i] - V, I);
    } else {
      for (int i = 0; i < P; i++) I = I + y[2 + npv * i];
    }
    R Vs;
    if (!cond && q.Delta_T == (R)0) Vs = (R)0;
    else Vs = q.Delta_T * (R)exp_m((float)((V - q.V_th) * q.inv_Delta_T));
    R s = fmaR(-q.g_L, (V - q.E_L) - Vs, I);
    s = s - w;
    s = s + q.I_e;
    dy[0] = (refr > (R)0) ? (R)0 : s * q.inv_C_m;
    dy[1] = fmaR(q.a, V - q.E_L, -w) * q.inv_tau_w;
    for (int i = 0; i < P; i++) {
      if (m == AEIF_COND_BETA) {
        dy[3 + 2 * i] = -y[3 + 2 * i] * q.inv_t1[i];
        dy[2 + 2 * i] = fmaR(-y[2 + 2 * i], q.inv_t2[i], y[3 + 2 * i]);
      } else if (m == AEIF_COND_ALPHA || m == AEIF_PSC_ALPHA) {
        dy[3 + 2 * i] = -y[3 + 2 * i] * q.inv_t1[i];
        dy[2 + 2 * i] = fmaR(-y[2 + 2 * i], q.inv_t1[i], y[3 + 2 * i]);
      } else {
        dy[2 + i] = -y[2 + i] * q.inv_t1[i];
      }
    }
  }

  template <class R> static R pow_dec(R err, bool f64) {
    if (f64) return (R)std::pow((double)err, -0.25);
    return (R)(1.0f / std::sqrt(std::sqrt((float)err)));
  }
  template <class R> static R pow_inc(R err, bool f64) {
    if (f64) return (R)std::pow((double)err, -0.2);
    return (R)exp_m(-0.2f * log_m((float)err));
  }

  // Error estimate (divided by the tolerance) of one FP32 trial step of size hh from y,
  // with the step's k1 and error scale: the trial arithmetic of rk5_step.
  template <class R>
  R trial_error(Model m, int P, int NV, const R *y, const R *k1, const R *iys, R hh, const Par<R> &q, R refr) {
    static const C5<R> K;
    R a[64] = {}, b2[64] = {}, b3[64] = {}, b4[64] = {}, b5[64] = {}, b6[64] = {};
    for (int i = 0; i < NV; i++) a[i] = fmaR(hh * K.a21, k1[i], y[i]);
    derivs<R>(m, P, a, b2, q, refr);
    for (int i = 0; i < NV; i++) a[i] = fmaR(hh * K.a32, b2[i], fmaR(hh * K.a31, k1[i], y[i]));
    derivs<R>(m, P, a, b3, q, refr);
    for (int i = 0; i < NV; i++) a[i] = fmaR(hh * K.a43, b3[i], fmaR(hh * K.a42, b2[i], fmaR(hh * K.a41, k1[i], y[i])));
    derivs<R>(m, P, a, b4, q, refr);
    for (int i = 0; i < NV; i++)
      a[i] = fmaR(hh * K.a54, b4[i], fmaR(hh * K.a53, b3[i], fmaR(hh * K.a52, b2[i], fmaR(hh * K.a51, k1[i], y[i]))));
    derivs<R>(m, P, a, b5, q, refr);
    for (int i = 0; i < NV; i++)
      a[i] = fmaR(hh * K.a65, b5[i],
                  fmaR(hh * K.a64, b4[i], fmaR(hh * K.a63, b3[i], fmaR(hh * K.a62, b2[i], fmaR(hh * K.a61, k1[i], y[i])))));
    derivs<R>(m, P, a, b6, q, refr);
    R e = 0;
    for (int i = 0; i < NV; i++) {
      R v = fmaR(hh * K.e6, b6[i], fmaR(hh * K.e5, b5[i], fmaR(hh * K.e4, b4[i], fmaR(hh * K.e3, b3[i], hh * K.e1 * k1[i]))));
      R av = std::fabs(v * iys[i]);
      e = (e > av) ? e : av;
    }
    return e * (R)1.0e6f;
  }

  // Largest step in [hmin, hmax] whose trial passes the error test (bisection in log h,
  // 30 halvings): what a perfect proposal would choose.  Analysis only.
  template <class R>
  R largest_passing_step(Model m, int P, int NV, const R *y, const R *k1, const R *iys, R hmin, R hmax,
                         const Par<R> &q, R refr) {
    if (trial_error<R>(m, P, NV, y, k1, iys, hmax, q, refr) <= (R)1) return hmax;
    R lo = hmin, hi = hmax;
    for (int it = 0; it < 30; it++) {
      const R mid = (R)std::sqrt((double)lo * (double)hi);
      if (trial_error<R>(m, P, NV, y, k1, iys, mid, q, refr) <= (R)1) lo = mid;
      else hi = mid;
    }
    return lo;
  }

  // One accepted RK5 step (src/rk5.h:69-159).  Returns derivative calls.
  template <class R>
  int rk5_step(Model m, int P, int NV, double &x, R *y, R &h, R hmin, R hmax, const Par<R> &q, R refr) {
    static const C5<R> K;
    R k1[64], k2[64], k3[64], k4[64], k5[64], k6[64], yn[64], ys[64], iys[64];
    int nd = 1;
    derivs<R>(m, P, y, k1, q, refr);
    for (int i = 0; i < NV; i++) {
      ys[i] = std::fabs(y[i]) + std::fabs(k1[i] * h) + K.scal_min;
      iys[i] = (R)1 / ys[i];
    }
    R err;
    const R hmin_acc = hmin * (R)(fp64 ? 1.00001 : (double)1.00001f);
    int trials = 0;
    // learned step size: features after k1; the network proposes the first trial h
    // when the plain h would not reach the end of the time step
    float feat[sm::NF];
    if (!fp64 && learn_mode == 3) h = largest_passing_step<R>(m, P, NV, y, k1, iys, hmin, hmax, q, refr);
    if (!fp64 && (learn_mode == 1 || (learn_mode == 2 && h < hmax))) {
      const int npv = (m == AEIF_PSC_EXP) ? 1 : 2;
      feat[0] = (float)y[0];
      feat[1] = (float)y[1];
      for (int p = 0; p < 4; p++) feat[2 + p] = (p < P) ? (float)y[2 + npv * p] : 0.0f;
      float sdg = 0.0f;
      for (int p = 0; p < P; p++) sdg = sdg + (float)k1[2 + npv * p];
      feat[6] = slog_f((float)k1[0]);
      feat[7] = slog_f(sdg);
      feat[8] = log_m((float)h);
      feat[9] = log_m((float)hmax);
      if (learn_mode == 2) {
        const float hp = mlp_propose_f(model.data(), feat);
        if (hp > 0.0f && hp <= 3.0e38f) {
          const float lo = model[sm::FLOOR] * (float)h;
          h = (R)((hp > lo) ? hp : lo);
        }
      }
    }
    for (;;) {
      if (h > hmax) h = hmax;
      if (h < hmin) h = hmin;
      if (fp64) {
        for (int i = 0; i < NV; i++) yn[i] = y[i] + h * K.a21 * k1[i];
        derivs<R>(m, P, yn, k2, q, refr);
        for (int i = 0; i < NV; i++) yn[i] = y[i] + h * (K.a31 * k1[i] + K.a32 * k2[i]);
        derivs<R>(m, P, yn, k3, q, refr);
        for (int i = 0; i < NV; i++) yn[i] = y[i] + h * (K.a41 * k1[i] + K.a42 * k2[i] + K.a43 * k3[i]);
        derivs<R>(m, P, yn, k4, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = y[i] + h * (K.a51 * k1[i] + K.a52 * k2[i] + K.a53 * k3[i] + K.a54 * k4[i]);
        derivs<R>(m, P, yn, k5, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = y[i] + h * (K.a61 * k1[i] + K.a62 * k2[i] + K.a63 * k3[i] + K.a64 * k4[i] + K.a65 * k5[i]);
        derivs<R>(m, P, yn, k6, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = y[i] + h * (K.a71 * k1[i] + K.a73 * k3[i] + K.a74 * k4[i] + K.a76 * k6[i]);
        err = 0;
        for (int i = 0; i < NV; i++) {
          R v = h * (K.e1 * k1[i] + K.e3 * k3[i] + K.e4 * k4[i] + K.e5 * k5[i] + K.e6 * k6[i]);
          v /= ys[i];
          R av = std::fabs(v);
          err = (err > av) ? err : av;
        }
        err /= K.eps;
      } else {
        const R b21 = h * K.a21, b31 = h * K.a31, b32 = h * K.a32, b41 = h * K.a41, b42 = h * K.a42,
                b43 = h * K.a43, b51 = h * K.a51, b52 = h * K.a52, b53 = h * K.a53, b54 = h * K.a54,
                b61 = h * K.a61, b62 = h * K.a62, b63 = h * K.a63, b64 = h * K.a64, b65 = h * K.a65,
                b71 = h * K.a71, b73 = h * K.a73, b74 = h * K.a74, b76 = h * K.a76, f1 = h * K.e1,
                f3 = h * K.e3, f4 = h * K.e4, f5 = h * K.e5, f6 = h * K.e6;
        for (int i = 0; i < NV; i++) yn[i] = fmaR(b21, k1[i], y[i]);
        derivs<R>(m, P, yn, k2, q, refr);
        for (int i = 0; i < NV; i++) yn[i] = fmaR(b32, k2[i], fmaR(b31, k1[i], y[i]));
        derivs<R>(m, P, yn, k3, q, refr);
        for (int i = 0; i < NV; i++) yn[i] = fmaR(b43, k3[i], fmaR(b42, k2[i], fmaR(b41, k1[i], y[i])));
        derivs<R>(m, P, yn, k4, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = fmaR(b54, k4[i], fmaR(b53, k3[i], fmaR(b52, k2[i], fmaR(b51, k1[i], y[i]))));
        derivs<R>(m, P, yn, k5, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = fmaR(b65, k5[i], fmaR(b64, k4[i], fmaR(b63, k3[i], fmaR(b62, k2[i], fmaR(b61, k1[i], y[i])))));
        derivs<R>(m, P, yn, k6, q, refr);
        for (int i = 0; i < NV; i++)
          yn[i] = fmaR(b76, k6[i], fmaR(b74, k4[i], fmaR(b73, k3[i], fmaR(b71, k1[i], y[i]))));
        err = 0;
        for (int i = 0; i < NV; i++) {
          R v = fmaR(f6, k6[i], fmaR(f5, k5[i], fmaR(f4, k4[i], fmaR(f3, k3[i], f1 * k1[i]))));
          R av = std::fabs(v * iys[i]);
          err = (err > av) ? err : av;
        }
        err = err * (R)1.0e6f;
      }
      nd += 5;
      trials++;
      if (err <= (R)1 || h <= hmin_acc || trials >= 100000) break;
      R hnew = h * K.coeff * pow_dec<R>(err, fp64);
      R h01 = (R)0.1 * h;
      if (fp64) h01 = (R)(0.1 * (double)h);
      h = (hnew > h01) ? hnew : h01;
    }
    if (!fp64 && learn_mode == 1) {
#pragma omp critical(steplog)
      {
        if (log_offered < log_cap) {
          for (int k = 0; k < sm::NF; k++) steplog.push_back(feat[k]);
          steplog.push_back((float)h);
          steplog.push_back((float)err);
        }
        log_offered++;
      }
    }
#pragma omp atomic
    n_rk5_steps++;
#pragma omp atomic
    n_rk5_trials += trials;
    x += (double)h;
    if (err > K.err_min) h = h * K.coeff * pow_inc<R>(err, fp64);
    else h = (R)5 * h;
    if (!(h == h)) h = hmin;   // a NaN step size would never terminate the next step
    for (int i = 0; i < NV; i++) y[i] = yn[i];
    return nd;
  }

  void push_spike(int node, float height, long long tidx) {
    Group &g = group_of(node);
    int i = node - g.i0;
    if (part_world > 1 && !injecting) {
#pragma omp critical(step_spikes)
      step_spikes.push_back({node, height});
    }
#pragma omp atomic
    n_spikes_total++;
    if (g.spike_count_on) g.spike_count[i]++;
    if (g.max_rec > 0) {
      if ((int)g.rec_times[i].size() < g.max_rec - 1) g.rec_times[i].push_back((float)neural_time);
    }
    // the spike reaches the node's own synapses at once, or den_delay steps later
    // (src/spike_buffer.cu:183-186, 279-281, 314-316)
    if (den_steps[node] == 0) {
      last_rev[node] = tidx;
    } else {
#pragma omp critical(rev_pending)
      rev_pending[tidx + den_steps[node]].push_back(node);
    }
    if (!conn[node].empty()) {
      std::vector<Queued> &q = queue[node];
      if ((int)q.size() >= max_spike_buffer) return;   // reference prints and drops
      q.insert(q.begin(), Queued{0, 0, height});
    }
  }

  template <class R>
  void update_aeif(Group &g, double x1, long long tidx) {
    ModelShape s = shape_of(g.model);
    int P = g.nport;
    int NV = 2 + s.n_port_var * P;
    R hmin = (R)(g.h_min_rel * dt);
    if (fp64) hmin = (R)((double)g.h_min_rel * (double)dt);
    long long nd_total = 0;
    const int i_lo = g.lo, i_hi = g.hi < 0 ? g.n : g.hi;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : nd_total)
    for (int i = i_lo; i < i_hi; i++) {
      Par<R> q;
      auto gp = [&](int j) { return (R)g.par[j][i]; };
      q.V_th = gp(A_V_th); q.Delta_T = gp(A_Delta_T); q.g_L = gp(A_g_L); q.E_L = gp(A_E_L);
      q.C_m = gp(A_C_m); q.a = gp(A_a); q.b = gp(A_b); q.tau_w = gp(A_tau_w); q.I_e = gp(A_I_e);
      q.V_peak = gp(A_V_peak); q.V_reset = gp(A_V_reset); q.t_ref = gp(A_t_ref);
      q.inv_Delta_T = (R)1 / q.Delta_T; q.inv_C_m = (R)1 / q.C_m; q.inv_tau_w = (R)1 / q.tau_w;
      for (int p = 0; p < P; p++) {
        int b = A_NSCAL + s.n_port_par * p;
        switch (g.model) {
        case AEIF_COND_BETA: q.E_rev[p] = gp(b + 0); q.t1[p] = gp(b + 1); q.t2[p] = gp(b + 2); break;
        case AEIF_COND_ALPHA: q.E_rev[p] = gp(b + 0); q.t1[p] = gp(b + 1); q.t2[p] = q.t1[p]; break;
        default: q.E_rev[p] = 0; q.t1[p] = gp(b + 0); q.t2[p] = q.t1[p]; break;
        }
        q.inv_t1[p] = (R)1 / q.t1[p];
        q.inv_t2[p] = (R)1 / q.t2[p];
      }
      R y[64];
      for (int v = 0; v < NV; v++) y[v] = (R)g.var[v][i];
      R refr = (R)g.par[A_refractory_step][i];
      double x = g.x[i];
      R h = (R)g.h[i];
      bool end = false;
      int guard = 0;
      while (!end) {
        R hmax = (R)(x1 - x);
        nd_total += rk5_step<R>(g.model, P, NV, x, y, h, hmin, hmax, q, refr);
        end = (x >= x1 - (double)hmin);
        if (++guard > 1000000) break;
        // ExternalUpdate (src/aeif_cond_beta_multisynapse_kernel.h:190-226)
        if (y[0] < (R)-1.0e3) { y[0] = q.V_reset; y[1] = 0; continue; }
        if (y[1] < (R)-1.0e6 || y[1] > (R)1.0e6) { y[0] = q.V_reset; y[1] = 0; continue; }
        if (refr > (R)0) {
          y[0] = q.V_reset;
          if (end) refr -= (R)1;
        } else if (y[0] >= q.V_peak) {
          push_spike(g.i0 + i, 1.0f, tidx);
          y[0] = q.V_reset;
          y[1] += q.b;
          float rs = std::round((float)q.t_ref / dt);
          if (fp64) rs = (float)std::round((double)q.t_ref / (double)dt);
          refr = (R)(int)rs;
          if (refr < (R)0) refr = 0;
        }
      }
      for (int v = 0; v < NV; v++) g.var[v][i] = (double)y[v];
      g.par[A_refractory_step][i] = (double)refr;
      g.x[i] = x;
      g.h[i] = (double)h;
    }
    n_derivs += nd_total;
  }

  template <class R> void update_iaf(Group &g, long long tidx) {
    const int i_lo = g.lo, i_hi = g.hi < 0 ? g.n : g.hi;
#pragma omp parallel for schedule(static)
    for (int i = i_lo; i < i_hi; i++) {
      R Iex = (R)g.var[I_I_syn_ex][i], Iin = (R)g.var[I_I_syn_in][i];
      R V = (R)g.var[I_V_m_rel][i], refr = (R)g.var[I_refractory_step][i];
      auto gp = [&](int j) { return (R)g.par[j][i]; };
      if (refr > (R)0) {
        refr -= (R)1;
      } else {
        if (fp64) V = V * gp(I_P22) + Iex * gp(I_P21ex) + Iin * gp(I_P21in) + gp(I_I_e) * gp(I_P20);
        else V = fmaR(gp(I_I_e), gp(I_P20), fmaR(Iin, gp(I_P21in), fmaR(Iex, gp(I_P21ex), V * gp(I_P22))));
      }
      Iex = Iex * gp(I_P11ex);
      Iin = Iin * gp(I_P11in);
      if (V >= gp(I_Theta_rel)) {
        push_spike(g.i0 + i, 1.0f, tidx);
        V = gp(I_V_reset_rel);
        float rs = std::round((float)gp(I_t_ref) / dt);
        if (fp64) rs = (float)std::round((double)gp(I_t_ref) / (double)dt);
        refr = (R)(int)rs;
      }
      g.var[I_I_syn_ex][i] = Iex; g.var[I_I_syn_in][i] = Iin;
      g.var[I_V_m_rel][i] = V; g.var[I_refractory_step][i] = refr;
    }
  }

  float record_value(const Rec &r) {
    Group &g = group_of(r.node);
    int i = r.node - g.i0;
    if (r.var == "spike") {
      std::vector<Queued> &q = queue[r.node];
      if (q.empty() || q[0].age != 0) return 0.0f;
      return q[0].height;
    }
    if (r.var == "spike_count") return (float)g.spike_count[i];
    int kind;
    int idx = locate(g, r.var, kind);
    if (idx < 0 || kind > 3) throw std::runtime_error("Unrecognized record variable " + r.var);
    return (float)slot(g, kind, idx, r.port)[i];
  }

  void write_records(float t) {
    if (recs.empty()) return;
    std::vector<float> row;
    row.push_back(t);
    for (auto &r : recs) row.push_back(record_value(r));
    rec_rows.push_back(row);
  }

  void start() {
    if (!calibrated) calibrate();
    if (first_sim) {
      write_records((float)neural_time);
      first_sim = false;
    }
    neur_t0 = neural_time;
    it = 0;
  }

  void step() {
    // 1. spike buffer update (src/spike_buffer.cu:247-317)
    struct Ev { int src; int grp; float height; };
    std::vector<Ev> events;
    const int nthr = omp_get_max_threads();
    std::vector<std::vector<Ev>> tev(nthr);
#pragma omp parallel for schedule(dynamic, 1024)
    for (size_t s = 0; s < queue.size(); s++) {
      std::vector<Queued> &q = queue[s];
      if (q.empty()) continue;
      std::vector<Ev> &ev = tev[omp_get_thread_num()];
      int ng = (int)conn[s].size();
      int Ns = (int)q.size();
      bool drop_oldest = false;
      for (int is = 0; is < Ns; is++) {
        Queued &e = q[is];
        if (e.cursor < ng && e.age == conn[s][e.cursor].delay) {
          ev.push_back({(int)s, e.cursor, e.height});
          e.cursor++;
        }
        if (is == Ns - 1 && e.cursor >= ng) drop_oldest = true;
        else e.age++;
      }
      if (drop_oldest) q.pop_back();
    }
    for (auto &v : tev) events.insert(events.end(), v.begin(), v.end());
    // 2. time
    neural_time = neur_t0 + (double)dt * (double)(it + 1);
    long long tidx = (long long)(int)std::round(neur_t0 / (double)dt) + it + 1;
    cur_tidx = tidx;
    // 2b. keep the 16-bit arrival stamps of plastic edges unambiguous
    //     (src/nestgpu.cu:490-498, src/rev_spike.cu:93-118)
    if (any_plastic && ((tidx & 0xffff) == 0x8000 || (tidx & 0xffff) == 0)) {
      const bool up = (tidx & 0xffff) == 0x8000;
      for (auto &v : conn)
        for (auto &dg : v)
          for (auto &e : dg.tg) {
            if (!e.syn) continue;
            if (up && e.stamp >= 0x8000) e.stamp = 0;
            if (!up && e.stamp < 0x8000) e.stamp = 0x8000;
          }
    }
    // 3. update
    for (auto &g : groups) {
      if (is_aeif(g.model)) {
        if (fp64) update_aeif<double>(g, neural_time, tidx);
        else update_aeif<float>(g, neural_time, tidx);
      } else if (g.model == IAF_PSC_EXP) {
        if (fp64) update_iaf<double>(g, tidx);
        else update_iaf<float>(g, tidx);
      } else if (g.model == PARROT) {
        // src/parrot_neuron.cu:60-82
        for (int i = g.lo; i < (g.hi < 0 ? g.n : g.hi); i++) {
          const float sh = (float)g.var[PR_input_spike_height][i];
          g.var[PR_V][i] = sh;
          if (sh != 0.0f) {
            const float height = g.par[PR_hold_spike_height][i] == 0.0 ? 1.0f : sh;
            g.var[PR_input_spike_height][i] = 0.0;
            push_spike(g.i0 + i, height, tidx);
          }
        }
      } else if (g.model == SPIKE_DET) {
        // src/spike_detector.cu:28-50
        for (int i = g.lo; i < (g.hi < 0 ? g.n : g.hi); i++) {
          float sh = (float)g.var[SD_input_spike_height][i];
          if (sh != 0.0f) {
            if (g.par[SD_hold_spike_height][i] == 0.0) sh = 1.0f;
            g.var[SD_input_spike_height][i] = 0.0;
          }
          g.var[SD_spike_height][i] = sh;
        }
      } else if (g.model == SPIKE_GEN) {
        for (int i = g.lo; i < (g.hi < 0 ? g.n : g.hi); i++) {
          int k = g.sg_next[i];
          if (k < (int)g.sg_tidx[i].size() && g.sg_tidx[i][k] == (int)it) {
            push_spike(g.i0 + i, g.sg_height[i][k], tidx);
            g.sg_next[i]++;
          }
        }
      }
    }
    // partitioned network: the spikes this process's neurons emitted in the step go to the
    // other processes, theirs come back and enter the per-source queues at this step, as if
    // emitted here (the exchange the engine makes once per time batch)
    if (part_world > 1) {
      if (!xch_fn || xch_fn(xch_user) != 0) throw std::runtime_error("the spike exchange failed");
      step_spikes.clear();
    }
    // 4. records
    write_records((float)neural_time);
    // 4b. reverse spikes whose dendritic delay ends in this step (set at the start of the
    //     step in the reference, src/spike_buffer.cu:314-316; only the plasticity below reads it)
    if (!rev_pending.empty()) {
      auto it = rev_pending.find(tidx);
      if (it != rev_pending.end()) {
        for (int nd : it->second) last_rev[nd] = tidx;
        rev_pending.erase(it);
      }
    }
    // 5. collect spikes (src/get_spike.cu:60-108); FP64 sums, order-independent for
    //    weights whose partial sums are exact
    long long nev = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : nev)
    for (size_t k = 0; k < events.size(); k++) {
      const Ev &ev = events[k];
      for (auto &e : conn[ev.src][ev.grp].tg) {
        Group &tg = groups[node_group[e.tgt]];
        double &a = tg.acc[(size_t)e.port * tg.n + (e.tgt - tg.i0)];
        double v = (double)(ev.height * e.w);
#pragma omp atomic
        a += v;
        nev++;
        if (e.syn) {
          // src/get_spike.cu:85-95: arrival stamp, depression against the target's last spike
          e.stamp = (unsigned short)(tidx & 0xffff);
          const long long Dt_int = tidx - last_rev[e.tgt];
          if (Dt_int > 0 && Dt_int < kMaxSynDt)
            e.w = synapse_update(syn_groups[e.syn - 1], e.w, -dt * (float)Dt_int);
        }
      }
    }
    n_events += nev;
    // 6. poiss_gen direct spikes (src/poiss_gen.cu:55-86)
    float time_step = (float)(dt / 1000.0);
#pragma omp parallel for schedule(static)
    for (size_t ie = 0; ie < direct.size(); ie++) {
      const Direct &d = direct[ie];
      const Group &g = groups[d.group];
      float rate = (float)g.par[PG_rate][d.gen], origin = (float)g.par[PG_origin][d.gen];
      float start_ = (float)g.par[PG_start][d.gen], stop_ = (float)g.par[PG_stop][d.gen];
      double t_rel = neural_time - (double)origin - (double)d.delay;
      if (t_rel >= (double)start_ && t_rel <= (double)stop_) {
        int n = poisson_draw(time_step * rate, kernel_seed, d.key, tidx);
        if (n > 0) {
          Group &tg = groups[node_group[d.tgt]];
          double &a = tg.acc[(size_t)d.port * tg.n + (d.tgt - tg.i0)];
          double v = (double)(d.w * (float)n);
#pragma omp atomic
          a += v;
        }
      }
    }
    // 7. fold inputs (src/get_spike.cu:142-166)
    for (auto &g : groups) {
      if (g.nport == 0) continue;
      ModelShape s = shape_of(g.model);
      for (int p = 0; p < g.nport; p++)
#pragma omp parallel for schedule(static)
        for (int i = 0; i < g.n; i++) {
          double a = g.acc[(size_t)p * g.n + i];
          if (a == 0.0) continue;
          g.acc[(size_t)p * g.n + i] = 0.0;
          double pw;
          std::vector<double> *pi;
          if (is_aeif(g.model)) {
            pw = s.weight_par >= 0 ? (double)(float)g.par[A_NSCAL + s.n_port_par * p + s.weight_par][i] : 1.0;
            pi = &g.var[2 + s.n_port_var * p + s.input_var];
          } else if (g.model == PARROT) {
            // port weights {1, 0}: port p feeds variable p (src/parrot_neuron.cu:110-122)
            pw = p == 0 ? 1.0 : 0.0;
            pi = &g.var[p];
          } else if (g.model == SPIKE_DET) {
            pw = 1.0;
            pi = &g.var[SD_input_spike_height];
          } else {
            pw = 1.0;
            pi = &g.var[p == 0 ? I_I_syn_ex : I_I_syn_in];
          }
          double cur = (*pi)[i];
          if (fp64) (*pi)[i] = std::fma(a, pw, cur);
          else (*pi)[i] = (double)(float)std::fma(a, pw, (double)(float)cur);
        }
    }
    // 8. reverse spikes (src/rev_spike.cu:46-92, src/nestgpu.cu:606-616): the plastic
    //    in-edges of every node that spiked in this step are potentiated
    if (any_plastic) {
      const unsigned short t16 = (unsigned short)(tidx & 0xffff);
#pragma omp parallel for schedule(dynamic, 64)
      for (size_t nd = 0; nd < rev_in.size(); nd++) {
        if (rev_in[nd].empty() || last_rev[nd] != tidx) continue;
        for (Edge *e : rev_in[nd]) {
          const unsigned short Dt_int = (unsigned short)(t16 - e->stamp);
          if (Dt_int < kMaxSynDt) e->w = synapse_update(syn_groups[e->syn - 1], e->w, dt * (float)Dt_int);
        }
      }
    }
    it++;
  }

  void simulate(float T) {
    start();
    Nt = (long long)std::round(T / dt);
    for (long long k = 0; k < Nt; k++) step();
  }
};

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI for the Python test harness (oracle/oracle.py)
// ---------------------------------------------------------------------------
using orc::Net;
using orc::SynGroupDef;
using orc::SYN_STDP;
using orc::SYN_TEST;
using orc::kStdpPar;
using orc::kTestPar;

static thread_local std::string g_err;

#define OR_TRY try {
#define OR_CATCH(ret)                         \
  }                                           \
  catch (std::exception & e) {                \
    g_err = e.what();                         \
    return ret;                               \
  }

extern "C" {

const char *orc_error() { return g_err.c_str(); }

void *orc_new(int fp64) {
  OR_TRY
  Net *n = new Net();
  n->fp64 = fp64 != 0;
  return n;
  OR_CATCH(nullptr)
}
void orc_delete(void *p) { delete (Net *)p; }

int orc_set_time_resolution(void *p, float dt) { ((Net *)p)->dt = dt; return 0; }
float orc_get_time_resolution(void *p) { return ((Net *)p)->dt; }
int orc_set_seed(void *p, unsigned long long s) {
  OR_TRY((Net *)p)->reseed(s); return 0; OR_CATCH(-1)
}
int orc_set_max_spike_buffer_size(void *p, int n) { ((Net *)p)->max_spike_buffer = n; return 0; }

int orc_create(void *p, const char *model, int n, int nport) {
  OR_TRY return ((Net *)p)->create(model, n, nport); OR_CATCH(-1)
}
int orc_n_nodes(void *p) { return (int)((Net *)p)->node_group.size(); }
int orc_node_model(void *p, int node) {
  OR_TRY return (int)((Net *)p)->group_of(node).model; OR_CATCH(-1)
}
int orc_node_nport(void *p, int node) {
  OR_TRY return ((Net *)p)->group_of(node).nport; OR_CATCH(-1)
}

// kind codes returned: 0 scal var, 1 port var, 2 scal param, 3 port param, 4 group, 5 array; -1 none
int orc_locate(void *p, int node, const char *name) {
  OR_TRY
  Net *n = (Net *)p;
  int kind = -1;
  int idx = n->locate(n->group_of(node), name, kind);
  return idx < 0 ? -1 : kind;
  OR_CATCH(-2)
}

int orc_set(void *p, int node, int count, const char *name, int port, const float *vals, int stride) {
  OR_TRY
  Net *n = (Net *)p;
  for (int i = 0; i < count; i++) n->set_value(node + i, name, port, vals[stride ? i : 0]);
  return 0;
  OR_CATCH(-1)
}
int orc_set_list(void *p, const int *nodes, int count, const char *name, int port, const float *vals, int stride) {
  OR_TRY
  Net *n = (Net *)p;
  for (int i = 0; i < count; i++) n->set_value(nodes[i], name, port, vals[stride ? i : 0]);
  return 0;
  OR_CATCH(-1)
}
int orc_get(void *p, int node, int count, const char *name, int port, float *out) {
  OR_TRY
  Net *n = (Net *)p;
  for (int i = 0; i < count; i++) out[i] = n->get_value(node + i, name, port);
  return 0;
  OR_CATCH(-1)
}
int orc_set_spike_times(void *p, int node, int ns, const float *t, const float *h) {
  OR_TRY((Net *)p)->set_spike_times(node, ns, t, h); return 0; OR_CATCH(-1)
}

int orc_random_int(void *p, size_t n, unsigned int *out) {
  OR_TRY auto v = ((Net *)p)->random_int(n); std::copy(v.begin(), v.end(), out); return 0; OR_CATCH(-1)
}
int orc_random_uniform(void *p, size_t n, float *out) {
  OR_TRY auto v = ((Net *)p)->random_uniform(n); std::copy(v.begin(), v.end(), out); return 0; OR_CATCH(-1)
}
int orc_random_normal(void *p, size_t n, float mean, float sd, float *out) {
  OR_TRY auto v = ((Net *)p)->random_normal(n, mean, sd); std::copy(v.begin(), v.end(), out); return 0; OR_CATCH(-1)
}
// out must hold (n/4+1)*4 values
int orc_random_normal_clipped(void *p, size_t n, float mean, float sd, float vmin, float vmax,
                              float vstep, float *out) {
  OR_TRY
  auto v = ((Net *)p)->random_normal_clipped(n, mean, sd, vmin, vmax, vstep);
  std::copy(v.begin(), v.end(), out);
  return 0;
  OR_CATCH(-1)
}

int orc_connect(void *p, int rule, const int *src, int src0, int ns, const int *tgt, int tgt0, int nt,
                int degree, int port, int syn, float w, float d, const float *warr, const float *darr) {
  OR_TRY
  ((Net *)p)->connect_rule(rule, src, src0, ns, tgt, tgt0, nt, degree, port, syn, w, d, warr, darr);
  return 0;
  OR_CATCH(-1)
}
int orc_connect1(void *p, int src, int tgt, int port, float w, float d) {
  OR_TRY((Net *)p)->connect1(src, tgt, port, w, d); return 0; OR_CATCH(-1)
}

// Synapse groups (src/syn_model.cu:136-238): 1-based indices, 0 is the static synapse.
int orc_create_syn_group(void *p, const char *model) {
  OR_TRY
  Net *n = (Net *)p;
  if (n->calibrated) throw std::runtime_error("Nodes cannot be created after calibration");
  const std::string m = model;
  SynGroupDef g;
  if (m == "test_syn_model") { g.type = SYN_TEST; g.par = {0.1f, 0.0f}; }
  else if (m == "stdp") { g.type = SYN_STDP; g.par = {20.0f, 20.0f, 1.0e-4f, 1.0f, 1.0f, 1.0f, 100.0f}; }
  else throw std::runtime_error("Unknown synapse model name: " + m);
  n->syn_groups.push_back(g);
  return (int)n->syn_groups.size();
  OR_CATCH(-1)
}
static int syn_par_idx(Net *n, int g, const char *name) {
  if (g < 1 || g > (int)n->syn_groups.size()) throw std::runtime_error("Unrecognized synapse group");
  const SynGroupDef &d = n->syn_groups[g - 1];
  const char *const *names = d.type == SYN_STDP ? kStdpPar : kTestPar;
  for (size_t i = 0; i < d.par.size(); i++)
    if (std::string(name) == names[i]) return (int)i;
  throw std::runtime_error(std::string("Unrecognized synapse parameter ") + name);
}
int orc_set_syn_param(void *p, int g, const char *name, float v) {
  OR_TRY Net *n = (Net *)p; n->syn_groups[g - 1].par[syn_par_idx(n, g, name)] = v; return 0; OR_CATCH(-1)
}
int orc_get_syn_param(void *p, int g, const char *name, float *v) {
  OR_TRY Net *n = (Net *)p; *v = n->syn_groups[g - 1].par[syn_par_idx(n, g, name)]; return 0; OR_CATCH(-1)
}

// ---- partitioned network (the engine's process partition, restated step by step)
int orc_set_partition(void *p, int rank, int world) {
  OR_TRY
  Net *n = (Net *)p;
  if (world < 1 || rank < 0 || rank >= world) throw std::runtime_error("partition rank out of range");
  n->part_rank = rank;
  n->part_world = world;
  return 0;
  OR_CATCH(-1)
}
int orc_set_exchange(void *p, int (*fn)(void *), void *user) {
  ((Net *)p)->xch_fn = fn;
  ((Net *)p)->xch_user = user;
  return 0;
}
// the spikes this process's neurons emitted in the current step (nodes / heights may be null
// to ask for the count)
int orc_step_spikes(void *p, int *nodes, float *heights) {
  Net *n = (Net *)p;
  if (nodes)
    for (size_t j = 0; j < n->step_spikes.size(); j++) {
      nodes[j] = n->step_spikes[j].node;
      heights[j] = n->step_spikes[j].height;
    }
  return (int)n->step_spikes.size();
}
// the other processes' spikes of the current step, filed as if emitted here
int orc_inject_spikes(void *p, const int *nodes, const float *heights, int count) {
  OR_TRY
  Net *n = (Net *)p;
  n->injecting = true;
  for (int j = 0; j < count; j++) n->push_spike(nodes[j], heights[j], n->cur_tidx);
  n->injecting = false;
  return 0;
  OR_CATCH(-1)
}
int orc_connect_generated(void *p, int src0, int ns, int tgt0, int nt, int k, int port, float w,
                          float dmin_ms, float dmax_ms, unsigned long long seed) {
  OR_TRY ((Net *)p)->connect_generated(src0, ns, tgt0, nt, k, port, w, dmin_ms, dmax_ms, seed); return 0;
  OR_CATCH(-1)
}
int orc_set_poisson_stream(void *p, int i0, int n, unsigned int stream0) {
  OR_TRY
  Net *net = (Net *)p;
  for (int j = 0; j < n; j++) {
    if (net->group_of(i0 + j).model != orc::POISS_GEN) throw std::runtime_error("not a poisson_generator");
    net->pg_stream[i0 + j] = stream0 + (uint32_t)j;
  }
  return 0;
  OR_CATCH(-1)
}
int orc_connect_arrays(void *p, size_t n, const int *src, const int *tgt, const int *port,
                       const float *w, const float *d) {
  OR_TRY
  Net *net = (Net *)p;
  for (size_t i = 0; i < n; i++) net->connect1(src[i], tgt[i], port[i], w[i], d[i]);
  return 0;
  OR_CATCH(-1)
}
// ---- learned step size
int orc_step_model_nparams() { return orc::sm::NPAR; }
int orc_log_start(void *p, long long cap) {
  OR_TRY
  Net &n = *(Net *)p;
  if (n.fp64) throw std::runtime_error("the learned step size needs the FP32 mode");
  n.learn_mode = 1;
  n.log_cap = cap;
  n.log_offered = 0;
  n.steplog.clear();
  return 0;
  OR_CATCH(-1)
}
int orc_set_bound_mode(void *p, int on) {
  OR_TRY
  Net &n = *(Net *)p;
  if (n.fp64) throw std::runtime_error("the step-size bound needs the FP32 mode");
  n.learn_mode = on ? 3 : 0;
  return 0;
  OR_CATCH(-1)
}
int orc_log_stop(void *p) {
  Net &n = *(Net *)p;
  if (n.learn_mode == 1) n.learn_mode = 0;
  return 0;
}
long long orc_log_count(void *p, long long *offered) {
  Net &n = *(Net *)p;
  if (offered) *offered = n.log_offered;
  return (long long)(n.steplog.size() / orc::sm::LOG_W);
}
int orc_log_get(void *p, float *out) {
  Net &n = *(Net *)p;
  std::copy(n.steplog.begin(), n.steplog.end(), out);
  return 0;
}
int orc_step_model_set(void *p, const float *params, int enable) {
  OR_TRY
  Net &n = *(Net *)p;
  if (n.fp64) throw std::runtime_error("the learned step size needs the FP32 mode");
  n.model.assign(params, params + orc::sm::NPAR);
  n.learn_mode = enable ? 2 : 0;
  return 0;
  OR_CATCH(-1)
}
void orc_mlp_out(const float *params, const float *feat, int n, float *out) {
  for (int s = 0; s < n; s++) out[s] = orc::mlp_out_f(params, feat + (size_t)s * orc::sm::NF);
}
void orc_mlp_propose(const float *params, const float *feat, int n, float *out) {
  for (int s = 0; s < n; s++) out[s] = orc::mlp_propose_f(params, feat + (size_t)s * orc::sm::NF);
}
double orc_mlp_grad(const float *params, const float *feat, const float *target, int n, double *grad) {
  return orc::mlp_grad_d(params, feat, target, n, grad);
}
double orc_mlp_grad_bf16(const float *params, const float *feat, const float *target, int n, double *grad) {
  return orc::mlp_grad_bf16_d(params, feat, target, n, grad);
}

int orc_threads() { return omp_get_max_threads(); }

long long orc_n_conn(void *p) {
  Net *n = (Net *)p;
  long long c = 0;
  for (auto &v : n->conn) for (auto &dg : v) c += (long long)dg.tg.size();
  return c;
}
// Connections in reference order: source ascending, delay group ascending, insertion order.
// Columns: source, group index, index in group, target, port, delay (ms), weight.
int orc_get_conns(void *p, int *src, int *grp, int *idx, int *tgt, int *port, int *syn, float *delay, float *w) {
  Net *n = (Net *)p;
  long long c = 0;
  for (size_t s = 0; s < n->conn.size(); s++)
    for (size_t g = 0; g < n->conn[s].size(); g++) {
      const auto &dg = n->conn[s][g];
      for (size_t k = 0; k < dg.tg.size(); k++) {
        src[c] = (int)s; grp[c] = (int)g; idx[c] = (int)k; tgt[c] = dg.tg[k].tgt;
        port[c] = dg.tg[k].port; syn[c] = dg.tg[k].syn; delay[c] = n->dt * (float)(dg.delay + 1);
        w[c] = dg.tg[k].w;
        c++;
      }
    }
  return 0;
}

int orc_record(void *p, int node, const char *var, int port) {
  Net *n = (Net *)p;
  n->recs.push_back({node, var, port});
  return (int)n->recs.size() - 1;
}
int orc_record_rows(void *p) { return (int)((Net *)p)->rec_rows.size(); }
int orc_record_data(void *p, float *out) {
  Net *n = (Net *)p;
  size_t c = 0;
  for (auto &r : n->rec_rows) for (float v : r) out[c++] = v;
  return 0;
}
int orc_activate_spike_count(void *p, int node, int count) {
  OR_TRY
  Net *n = (Net *)p;
  orc::Group &g = n->group_of(node);
  g.spike_count_on = true;
  g.spike_count.assign(g.n, 0);
  (void)count;
  return 0;
  OR_CATCH(-1)
}
int orc_activate_rec_spike_times(void *p, int node, int count, int max_n) {
  OR_TRY
  Net *n = (Net *)p;
  orc::Group &g = n->group_of(node);
  g.max_rec = max_n;
  g.rec_times.assign(g.n, {});
  (void)count;
  return 0;
  OR_CATCH(-1)
}
int orc_get_spike_count(void *p, int node, int count, int *out) {
  OR_TRY
  Net *n = (Net *)p;
  for (int i = 0; i < count; i++) {
    orc::Group &g = n->group_of(node + i);
    out[i] = g.spike_count_on ? g.spike_count[node + i - g.i0] : 0;
  }
  return 0;
  OR_CATCH(-1)
}
int orc_n_rec_spike_times(void *p, int node) {
  OR_TRY
  Net *n = (Net *)p;
  orc::Group &g = n->group_of(node);
  return (int)g.rec_times[node - g.i0].size();
  OR_CATCH(-1)
}
int orc_rec_spike_times(void *p, int node, float *out) {
  OR_TRY
  Net *n = (Net *)p;
  orc::Group &g = n->group_of(node);
  auto &v = g.rec_times[node - g.i0];
  std::copy(v.begin(), v.end(), out);
  return 0;
  OR_CATCH(-1)
}

int orc_calibrate(void *p) { OR_TRY((Net *)p)->calibrate(); return 0; OR_CATCH(-1) }
int orc_simulate(void *p, float T) { OR_TRY((Net *)p)->simulate(T); return 0; OR_CATCH(-1) }
long long orc_n_derivs(void *p) { return ((Net *)p)->n_derivs; }
long long orc_n_rk5_steps(void *p) { return ((Net *)p)->n_rk5_steps; }
long long orc_n_rk5_trials(void *p) { return ((Net *)p)->n_rk5_trials; }
long long orc_n_spikes(void *p) { return ((Net *)p)->n_spikes_total; }
long long orc_n_events(void *p) { return ((Net *)p)->n_events; }
double orc_neural_time(void *p) { return ((Net *)p)->neural_time; }

// Standalone math probes (for unit tests of the own exp/log and the samplers).
float orc_exp_m(float x) { return orc::exp_m(x); }
float orc_log_m(float x) { return orc::log_m(x); }
int orc_poisson_draw(float lam, unsigned long long seed, unsigned long long edge, long long tidx) {
  return orc::poisson_draw(lam, seed, edge, tidx);
}
void orc_philox(unsigned int c0, unsigned int c1, unsigned int c2, unsigned int c3, unsigned int k0,
                unsigned int k1, unsigned int *out) {
  orc::U4 r = orc::philox({c0, c1, c2, c3}, k0, k1);
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

}  // extern "C"
