// CUDA kernels of the spiking engine (sm_100a).
//
// Per time step the host graph runs, in order:
//   1. one update kernel per node group (aeif RK5 / iaf_psc_exp / spike_generator);
//      each neuron first folds the inputs that arrived at the end of the previous
//      step (delivered spikes in the FP64 accumulator plus that step's poiss_gen
//      draws), then integrates one step and appends its spikes to the ring slot
//      of this step;
//   2. the record gather (when records exist);
//   3. the delivery kernel: the spikes emitted D steps ago walk their CSR segment
//      of delay D and add height*weight into the accumulator with FP64 atomics.
// This reproduces the reference order (src/nestgpu.cu:469-635): spike-buffer
// update, neuron update, record, CollectSpike, poiss_gen, GetSpikes fold.
#include <cub/block/block_scan.cuh>

#include <algorithm>

#include "ngpu_math.cuh"
#include "ngpu_types.h"

namespace ngpu {

// Cash-Karp tableau and controller constants (src/rk5.cu:35-72), FP32.
namespace ck {
constexpr float a21 = (float)0.2, a31 = (float)(3.0 / 40.0), a32 = (float)(9.0 / 40.0);
constexpr float a41 = (float)0.3, a42 = (float)-0.9, a43 = (float)1.2;
constexpr float a51 = (float)(-11.0 / 54.0), a52 = (float)2.5, a53 = (float)(-70.0 / 27.0),
                a54 = (float)(35.0 / 27.0);
constexpr float a61 = (float)(1631.0 / 55296.0), a62 = (float)(175.0 / 512.0),
                a63 = (float)(575.0 / 13824.0), a64 = (float)(44275.0 / 110592.0),
                a65 = (float)(253.0 / 4096.0);
constexpr float a71 = (float)(37.0 / 378.0), a73 = (float)(250.0 / 621.0),
                a74 = (float)(125.0 / 594.0), a76 = (float)(512.0 / 1771.0);
constexpr float e1 = (float)(37.0 / 378.0 - 2825.0 / 27648.0),
                e3 = (float)(250.0 / 621.0 - 18575.0 / 48384.0),
                e4 = (float)(125.0 / 594.0 - 13525.0 / 55296.0), e5 = (float)(-277.00 / 14336.0),
                e6 = (float)(512.0 / 1771.0 - 0.25);
constexpr float coeff = (float)0.9, err_min = (float)1.889568e-4, scal_min = (float)1.0e-1;
constexpr float inv_eps = 1.0e6f;
constexpr int max_trials = 100000;
constexpr int max_substeps = 1000000;
}  // namespace ck

__device__ __forceinline__ void step_time(const Clock *c, int k, float dt, long long &it,
                                          long long &tidx, double &tnow) {
  it = c->it0 + k;
  tidx = c->tidx_base + it + 1;
  tnow = c->t0 + (double)dt * (double)(it + 1);
}

// PushSpike (src/spike_buffer.cu:162-242) on the ring design.
__device__ __forceinline__ void push_spike(const SpikeOut &so, const GroupSpikeRec &rec, int node,
                                           int rel, float height, long long tidx, double tnow) {
  so.last_tidx[node] = (int)tidx;
  so.last_height[node] = height;
  atomicAdd(so.n_spikes, 1ULL);
  if (rec.spike_count) rec.spike_count[rel] += 1;
  if (rec.n_rec) {
    int nr = rec.n_rec[rel];
    if (nr < rec.max_rec - 1) {
      rec.rec_times[(size_t)rel * rec.max_rec + nr] = (float)tnow;
      rec.n_rec[rel] = nr + 1;
    } else {
      atomicOr(so.status, ST_REC_TIMES_FULL);
    }
  }
  if (so.has_out[node]) {
    int slot = (int)(tidx % so.R);
    int pos = atomicAdd(&so.ring_cnt[slot], 1);
    if (pos < so.cap) so.ring[(size_t)slot * so.cap + pos] = make_int2(node, __float_as_int(height));
    else atomicOr(so.status, ST_RING_OVERFLOW);
  }
}

// Input of the previous step for neuron i: accumulator plus poiss_gen draws
// (src/get_spike.cu:142-166, src/poiss_gen.cu:55-86).  `in` has nport entries.
__device__ __forceinline__ void gather_inputs(double *in, int nport, int n, int i, double *acc,
                                              const int *pin_off, const PoissonIn *pin,
                                              const GenPar *gen, float lam_scale, uint64_t seed,
                                              long long tidx_prev, double t_prev) {
  for (int p = 0; p < nport; p++) {
    double a = acc[(size_t)p * n + i];
    in[p] = a;
    if (a != 0.0) acc[(size_t)p * n + i] = 0.0;
  }
  if (pin_off) {
    int e0 = pin_off[i], e1 = pin_off[i + 1];
    for (int e = e0; e < e1; e++) {
      PoissonIn pe = pin[e];
      GenPar g = gen[pe.gen];
      double t_rel = t_prev - (double)g.origin - (double)pe.delay;
      if (t_rel >= (double)g.start && t_rel <= (double)g.stop) {
        int k = poisson_draw(__fmul_rn(lam_scale, g.rate), seed, pe.edge_id, tidx_prev);
        if (k > 0) in[pe.port] += (double)__fmul_rn(pe.weight, (float)k);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// aeif_*_multisynapse: adaptive Cash-Karp RK5 (src/rk5.h:69-207)
// ---------------------------------------------------------------------------
template <int MODEL> struct AeifShape {
  static constexpr int npv = (MODEL == M_AEIF_PSC_EXP) ? 1 : 2;   // port vars per port
  static constexpr int in_var = (MODEL == M_AEIF_PSC_EXP) ? 0 : 1; // port var receiving input
  static constexpr bool cond = (MODEL == M_AEIF_COND_BETA || MODEL == M_AEIF_COND_ALPHA);
};

template <int MODEL, int P> struct AeifQ {
  float V_th, Delta_T, inv_Delta_T, g_L, E_L, inv_C_m, a, b, inv_tau_w, I_e, V_peak, V_reset,
      refr_steps;
  float E_rev[P], inv_t1[P], inv_t2[P], pw[P];
};

template <int MODEL, int P>
__device__ __forceinline__ void aeif_derivs(const float *y, float *dy, const AeifQ<MODEL, P> &q,
                                            float refr) {
  typedef AeifShape<MODEL> S;
  const float V = (refr > 0.0f) ? q.V_reset : ((y[0] < q.V_peak) ? y[0] : q.V_peak);
  const float w = y[1];
  float I = 0.0f;
#pragma unroll
  for (int i = 0; i < P; i++) {
    if (S::cond) I = __fmaf_rn(y[2 + 2 * i], __fsub_rn(q.E_rev[i], V), I);
    else I = __fadd_rn(I, y[2 + S::npv * i]);
  }
  float Vs;
  if (!S::cond && q.Delta_T == 0.0f) Vs = 0.0f;
  else Vs = __fmul_rn(q.Delta_T, exp_m(__fmul_rn(__fsub_rn(V, q.V_th), q.inv_Delta_T)));
  float s = __fmaf_rn(-q.g_L, __fsub_rn(__fsub_rn(V, q.E_L), Vs), I);
  s = __fsub_rn(s, w);
  s = __fadd_rn(s, q.I_e);
  dy[0] = (refr > 0.0f) ? 0.0f : __fmul_rn(s, q.inv_C_m);
  dy[1] = __fmul_rn(__fmaf_rn(q.a, __fsub_rn(V, q.E_L), -w), q.inv_tau_w);
#pragma unroll
  for (int i = 0; i < P; i++) {
    if (MODEL == M_AEIF_PSC_EXP) {
      dy[2 + i] = __fmul_rn(-y[2 + i], q.inv_t1[i]);
    } else {
      dy[3 + 2 * i] = __fmul_rn(-y[3 + 2 * i], q.inv_t1[i]);
      dy[2 + 2 * i] = __fmaf_rn(-y[2 + 2 * i], q.inv_t2[i], y[3 + 2 * i]);
    }
  }
}

__device__ __forceinline__ float pget(const AeifArgs &A, int j, int i) {
  const float *p = A.parr[j];
  return p ? __ldg(p + i) : A.pval[j];
}

template <int MODEL, int P>
__device__ __forceinline__ void load_aeif_par(const AeifArgs &A, int i, AeifQ<MODEL, P> &q) {
  q.V_th = pget(A, AP_V_th, i);
  q.Delta_T = pget(A, AP_Delta_T, i);
  q.inv_Delta_T = pget(A, AP_inv_Delta_T, i);
  q.g_L = pget(A, AP_g_L, i);
  q.E_L = pget(A, AP_E_L, i);
  q.inv_C_m = pget(A, AP_inv_C_m, i);
  q.a = pget(A, AP_a, i);
  q.b = pget(A, AP_b, i);
  q.inv_tau_w = pget(A, AP_inv_tau_w, i);
  q.I_e = pget(A, AP_I_e, i);
  q.V_peak = pget(A, AP_V_peak, i);
  q.V_reset = pget(A, AP_V_reset, i);
  q.refr_steps = pget(A, AP_refr_steps, i);
#pragma unroll
  for (int p = 0; p < P; p++) {
    const int b = AEIF_NSCAL + AEIF_NPORTPAR * p;
    q.E_rev[p] = pget(A, b + 0, i);
    q.inv_t1[p] = pget(A, b + 1, i);
    q.inv_t2[p] = pget(A, b + 2, i);
    q.pw[p] = pget(A, b + 3, i);
  }
}

// One accepted RK5 step; returns the number of derivative evaluations.
template <int MODEL, int P>
__device__ __forceinline__ int rk5_step(double &x, float *y, float &h, float hmin, float hmin_acc,
                                        float hmax, const AeifQ<MODEL, P> &q, float refr,
                                        unsigned *status) {
  constexpr int NV = 2 + AeifShape<MODEL>::npv * P;
  float k1[NV], k2[NV], k3[NV], k4[NV], k5[NV], k6[NV], yn[NV], iys[NV];
  aeif_derivs<MODEL, P>(y, k1, q, refr);
#pragma unroll
  for (int i = 0; i < NV; i++) {
    float ys = __fadd_rn(__fadd_rn(fabsf(y[i]), fabsf(__fmul_rn(k1[i], h))), ck::scal_min);
    iys[i] = __fdiv_rn(1.0f, ys);
  }
  int nd = 1;
  int trials = 0;
  float err;
  for (;;) {
    if (h > hmax) h = hmax;
    if (h < hmin) h = hmin;
    const float b21 = __fmul_rn(h, ck::a21), b31 = __fmul_rn(h, ck::a31), b32 = __fmul_rn(h, ck::a32),
                b41 = __fmul_rn(h, ck::a41), b42 = __fmul_rn(h, ck::a42), b43 = __fmul_rn(h, ck::a43),
                b51 = __fmul_rn(h, ck::a51), b52 = __fmul_rn(h, ck::a52), b53 = __fmul_rn(h, ck::a53),
                b54 = __fmul_rn(h, ck::a54), b61 = __fmul_rn(h, ck::a61), b62 = __fmul_rn(h, ck::a62),
                b63 = __fmul_rn(h, ck::a63), b64 = __fmul_rn(h, ck::a64), b65 = __fmul_rn(h, ck::a65),
                b71 = __fmul_rn(h, ck::a71), b73 = __fmul_rn(h, ck::a73), b74 = __fmul_rn(h, ck::a74),
                b76 = __fmul_rn(h, ck::a76), f1 = __fmul_rn(h, ck::e1), f3 = __fmul_rn(h, ck::e3),
                f4 = __fmul_rn(h, ck::e4), f5 = __fmul_rn(h, ck::e5), f6 = __fmul_rn(h, ck::e6);
#pragma unroll
    for (int i = 0; i < NV; i++) yn[i] = __fmaf_rn(b21, k1[i], y[i]);
    aeif_derivs<MODEL, P>(yn, k2, q, refr);
#pragma unroll
    for (int i = 0; i < NV; i++) yn[i] = __fmaf_rn(b32, k2[i], __fmaf_rn(b31, k1[i], y[i]));
    aeif_derivs<MODEL, P>(yn, k3, q, refr);
#pragma unroll
    for (int i = 0; i < NV; i++)
      yn[i] = __fmaf_rn(b43, k3[i], __fmaf_rn(b42, k2[i], __fmaf_rn(b41, k1[i], y[i])));
    aeif_derivs<MODEL, P>(yn, k4, q, refr);
#pragma unroll
    for (int i = 0; i < NV; i++)
      yn[i] = __fmaf_rn(b54, k4[i],
                        __fmaf_rn(b53, k3[i], __fmaf_rn(b52, k2[i], __fmaf_rn(b51, k1[i], y[i]))));
    aeif_derivs<MODEL, P>(yn, k5, q, refr);
#pragma unroll
    for (int i = 0; i < NV; i++)
      yn[i] = __fmaf_rn(
          b65, k5[i],
          __fmaf_rn(b64, k4[i], __fmaf_rn(b63, k3[i], __fmaf_rn(b62, k2[i], __fmaf_rn(b61, k1[i], y[i])))));
    aeif_derivs<MODEL, P>(yn, k6, q, refr);
#pragma unroll
    for (int i = 0; i < NV; i++)
      yn[i] = __fmaf_rn(b76, k6[i],
                        __fmaf_rn(b74, k4[i], __fmaf_rn(b73, k3[i], __fmaf_rn(b71, k1[i], y[i]))));
    err = 0.0f;
#pragma unroll
    for (int i = 0; i < NV; i++) {
      float v = __fmaf_rn(f6, k6[i],
                          __fmaf_rn(f5, k5[i], __fmaf_rn(f4, k4[i], __fmaf_rn(f3, k3[i], __fmul_rn(f1, k1[i])))));
      float av = fabsf(__fmul_rn(v, iys[i]));
      err = (err > av) ? err : av;
    }
    err = __fmul_rn(err, ck::inv_eps);
    nd += 5;
    trials++;
    if (err <= 1.0f || h <= hmin_acc) break;
    if (trials >= ck::max_trials) {
      atomicOr(status, ST_RK5_TRIALS);
      break;
    }
    float hnew = __fmul_rn(__fmul_rn(h, ck::coeff), __fdiv_rn(1.0f, __fsqrt_rn(__fsqrt_rn(err))));
    float h01 = __fmul_rn(0.1f, h);
    h = (hnew > h01) ? hnew : h01;
  }
  x += (double)h;
  if (err > ck::err_min) h = __fmul_rn(__fmul_rn(h, ck::coeff), exp_m(__fmul_rn(-0.2f, log_m(err))));
  else h = __fmul_rn(5.0f, h);
  if (!(h == h)) h = hmin;
#pragma unroll
  for (int i = 0; i < NV; i++) y[i] = yn[i];
  return nd;
}

// RK5 steps of neuron i from x towards tnow (src/rk5.h:161-174), each followed by the
// model's ExternalUpdate.  Stops after `budget` steps (0: no limit); returns true when
// the neuron reached the end of the time step.
template <int MODEL, int P>
__device__ __forceinline__ bool aeif_integrate(const AeifArgs &A, const SpikeOut &so, int i,
                                               const AeifQ<MODEL, P> &q, float *y, float &refr,
                                               double &x, float &h, long long tidx, double tnow,
                                               int budget, unsigned long long &nd_acc) {
  const double x1 = tnow;
  bool end = false;
  int guard = 0, steps = 0;
  unsigned long long nd = 0;
  while (!end) {
    if (budget > 0 && steps == budget) {
      nd_acc += nd;
      return false;
    }
    float hmax = (float)(x1 - x);
    nd += rk5_step<MODEL, P>(x, y, h, A.hmin, A.hmin_acc, hmax, q, refr, so.status);
    steps++;
    end = (x >= x1 - (double)A.hmin);
    if (++guard > ck::max_substeps) {
      atomicOr(so.status, ST_RK5_TRIALS);
      break;
    }
    // ExternalUpdate (src/aeif_cond_beta_multisynapse_kernel.h:190-226)
    if (y[0] < -1.0e3f) {
      y[0] = q.V_reset;
      y[1] = 0.0f;
      atomicOr(so.status, ST_NUMERIC);
      continue;
    }
    if (y[1] < -1.0e6f || y[1] > 1.0e6f) {
      y[0] = q.V_reset;
      y[1] = 0.0f;
      atomicOr(so.status, ST_NUMERIC);
      continue;
    }
    if (refr > 0.0f) {
      y[0] = q.V_reset;
      if (end) refr = __fsub_rn(refr, 1.0f);
    } else if (y[0] >= q.V_peak) {
      push_spike(so, A.rec, A.i0 + i, i, 1.0f, tidx, tnow);
      y[0] = q.V_reset;
      y[1] = __fadd_rn(y[1], q.b);
      refr = q.refr_steps;
    }
  }
  nd_acc += nd;
  return true;
}

// One neuron, one step.  FLUSH: only fold the pending inputs.
template <int MODEL, int P, bool FLUSH>
__device__ __forceinline__ void aeif_neuron(const AeifArgs &A, const SpikeOut &so, int i,
                                            long long tidx, double tnow, long long tidx_prev,
                                            double t_prev, bool pending, int *strag_cnt,
                                            unsigned long long &nd_acc) {
  typedef AeifShape<MODEL> S;
  constexpr int NV = 2 + S::npv * P;
  const int n = A.n;
  AeifQ<MODEL, P> q;
  load_aeif_par<MODEL, P>(A, i, q);
  float y[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) y[v] = A.var[(size_t)v * n + i];
  if (pending) {
    double in[P];
    gather_inputs(in, P, n, i, A.acc, A.pin_off, A.pin, A.gen, A.lam_scale, A.seed, tidx_prev,
                  t_prev);
#pragma unroll
    for (int p = 0; p < P; p++) {
      if (in[p] != 0.0) {
        const int iv = 2 + S::npv * p + S::in_var;
        y[iv] = (float)__fma_rn(in[p], (double)q.pw[p], (double)y[iv]);
      }
    }
  }
  if (FLUSH) {
    if (pending) {
#pragma unroll
      for (int p = 0; p < P; p++) {
        const int iv = 2 + S::npv * p + S::in_var;
        A.var[(size_t)iv * n + i] = y[iv];
      }
    }
    return;
  }
  float refr = A.refr[i];
  double x = A.x[i];
  float h = A.h[i];
  const bool done = aeif_integrate<MODEL, P>(A, so, i, q, y, refr, x, h, tidx, tnow, A.budget, nd_acc);
#pragma unroll
  for (int v = 0; v < NV; v++) A.var[(size_t)v * n + i] = y[v];
  A.refr[i] = refr;
  A.x[i] = x;
  A.h[i] = h;
  if (!done) {
    // more RK5 steps needed than the budget allows: the straggler kernel finishes it
    int pos = atomicAdd(strag_cnt, 1);
    A.strag_list[pos] = i;
  }
}

// Step timing of an update/flush launch.  Update: step `it` integrates to tnow and
// folds the inputs of step it-1.  Flush (after the last step of a call, when it0
// was already advanced past it): folds the inputs of that last step.
struct StepT {
  long long it, tidx, tidx_prev;
  double tnow, t_prev;
};

template <bool FLUSH>
__device__ __forceinline__ StepT step_times(const Clock *c, int k, float dt) {
  StepT s;
  step_time(c, k, dt, s.it, s.tidx, s.tnow);
  if (FLUSH) {
    s.it -= 1;
    s.tidx -= 1;
    s.tnow = c->t0 + (double)dt * (double)(s.it + 1);
    s.tidx_prev = s.tidx;
    s.t_prev = s.tnow;
  } else {
    s.tidx_prev = s.tidx - 1;
    s.t_prev = c->t0 + (double)dt * (double)s.it;
  }
  return s;
}

template <int MODEL, int P, bool FLUSH>
__global__ void __launch_bounds__(128) aeif_update_kernel(const AeifArgs A, const SpikeOut so,
                                                          Clock *clk, int k) {
  const StepT t = step_times<FLUSH>(clk, k, A.dt);
  const bool pending = clk->pending != 0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nd = 0;
  if (i < A.n)
    aeif_neuron<MODEL, P, FLUSH>(A, so, i, t.tidx, t.tnow, t.tidx_prev, t.t_prev, pending,
                                 A.strag_cnt + (t.it & 1), nd);
  if (!FLUSH) {
    // one counter update per warp
    for (int o = 16; o > 0; o >>= 1) nd += __shfl_down_sync(0xffffffffu, nd, o);
    if ((threadIdx.x & 31) == 0 && nd) atomicAdd(A.nderiv, nd);
  }
}

// Neurons that needed more RK5 steps than the main kernel's budget (typically the
// few that spike in this step) finish here, packed densely into warps, so that their
// long step sequences no longer stall 31 idle lanes each.  The list of step `it` is
// indexed by its parity; the other parity's counter is cleared for the next step.
template <int MODEL, int P>
__global__ void __launch_bounds__(128) aeif_straggler_kernel(const AeifArgs A, const SpikeOut so,
                                                             Clock *clk, int k) {
  constexpr int NV = 2 + AeifShape<MODEL>::npv * P;
  const StepT t = step_times<false>(clk, k, A.dt);
  const int par = (int)(t.it & 1);
  const int cnt = A.strag_cnt[par];
  if (blockIdx.x == 0 && threadIdx.x == 0) A.strag_cnt[par ^ 1] = 0;
  unsigned long long nd = 0;
  const int n = A.n;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
    const int i = A.strag_list[j];
    AeifQ<MODEL, P> q;
    load_aeif_par<MODEL, P>(A, i, q);
    float y[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) y[v] = A.var[(size_t)v * n + i];
    float refr = A.refr[i];
    double x = A.x[i];
    float h = A.h[i];
    aeif_integrate<MODEL, P>(A, so, i, q, y, refr, x, h, t.tidx, t.tnow, 0, nd);
#pragma unroll
    for (int v = 0; v < NV; v++) A.var[(size_t)v * n + i] = y[v];
    A.refr[i] = refr;
    A.x[i] = x;
    A.h[i] = h;
  }
  for (int o = 16; o > 0; o >>= 1) nd += __shfl_down_sync(0xffffffffu, nd, o);
  if ((threadIdx.x & 31) == 0 && nd) atomicAdd(A.nderiv, nd);
}

// Generic port count (P > MAX_TPL_PORT): ports handled with runtime loops over
// MAX_PORT-sized arrays.  Same arithmetic, slower (local memory).
template <int MODEL, bool FLUSH>
__global__ void __launch_bounds__(128) aeif_update_kernel_gen(const AeifArgs A, const SpikeOut so,
                                                              Clock *clk, int k);

// ---------------------------------------------------------------------------
// iaf_psc_exp exact propagator (src/iaf_psc_exp.cu:85-110)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float iget(const IafArgs &A, int j, int i) {
  const float *p = A.parr[j];
  return p ? __ldg(p + i) : A.pval[j];
}

template <bool FLUSH>
__global__ void __launch_bounds__(256) iaf_update_kernel(const IafArgs A, const SpikeOut so,
                                                         Clock *clk, int k, float dt) {
  const StepT t = step_times<FLUSH>(clk, k, dt);
  const long long tidx = t.tidx;
  const double tnow = t.tnow;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int n = A.n;
  float Iex = A.var[i], Iin = A.var[(size_t)n + i], V = A.var[2 * (size_t)n + i],
        refr = A.var[3 * (size_t)n + i];
  if (clk->pending) {
    double in[2];
    gather_inputs(in, 2, n, i, A.acc, A.pin_off, A.pin, A.gen, A.lam_scale, A.seed, t.tidx_prev,
                  t.t_prev);
    if (in[0] != 0.0) Iex = (float)__fma_rn(in[0], 1.0, (double)Iex);
    if (in[1] != 0.0) Iin = (float)__fma_rn(in[1], 1.0, (double)Iin);
  }
  if (FLUSH) {
    A.var[i] = Iex;
    A.var[(size_t)n + i] = Iin;
    return;
  }
  if (refr > 0.0f) {
    refr = __fsub_rn(refr, 1.0f);
  } else {
    V = __fmaf_rn(iget(A, IP_I_e, i), iget(A, IP_P20, i),
                  __fmaf_rn(Iin, iget(A, IP_P21in, i),
                            __fmaf_rn(Iex, iget(A, IP_P21ex, i), __fmul_rn(V, iget(A, IP_P22, i)))));
  }
  Iex = __fmul_rn(Iex, iget(A, IP_P11ex, i));
  Iin = __fmul_rn(Iin, iget(A, IP_P11in, i));
  if (V >= iget(A, IP_Theta_rel, i)) {
    push_spike(so, A.rec, A.i0 + i, i, 1.0f, tidx, tnow);
    V = iget(A, IP_V_reset_rel, i);
    refr = iget(A, IP_refr_steps, i);
  }
  A.var[i] = Iex;
  A.var[(size_t)n + i] = Iin;
  A.var[2 * (size_t)n + i] = V;
  A.var[3 * (size_t)n + i] = refr;
}

// ---------------------------------------------------------------------------
// spike_generator (src/spike_generator.cu:49-67): compares against the per-call
// step counter, at most one spike per step.
// ---------------------------------------------------------------------------
__global__ void spike_gen_kernel(const SpikeGenArgs A, const SpikeOut so, Clock *clk, int k,
                                 float dt) {
  long long it, tidx;
  double tnow;
  step_time(clk, k, dt, it, tidx, tnow);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  int e = A.off[i] + A.next[i];
  if (e < A.off[i + 1] && (long long)A.tidx[e] == it) {
    push_spike(so, A.rec, A.i0 + i, i, A.height[e], tidx, tnow);
    A.next[i] += 1;
  }
}

// ---------------------------------------------------------------------------
// Delivery: ring slots of the last dspan steps -> CSR segments -> FP64 atomics.
// One warp per (source, delay) event, lanes stride over the segment.
// ---------------------------------------------------------------------------
constexpr int DELIVER_THREADS = 256;
constexpr int MAX_DSPAN = 8192;

__global__ void __launch_bounds__(DELIVER_THREADS) deliver_kernel(const DeliverArgs A, Clock *clk,
                                                                  int k, float dt) {
  extern __shared__ int s_pref[];   // dspan + 1 prefix sums
  typedef cub::BlockScan<int, DELIVER_THREADS> Scan;
  __shared__ typename Scan::TempStorage scan_tmp;
  long long it, tidx;
  double tnow;
  step_time(clk, k, dt, it, tidx, tnow);
  const int dspan = A.dspan;
  const int per = (dspan + DELIVER_THREADS - 1) / DELIVER_THREADS;
  int local = 0;
  const int b0 = threadIdx.x * per;
  for (int j = 0; j < per; j++) {
    int dd = b0 + j;
    if (dd < dspan) {
      long long ts = tidx - 1 - (A.dmin + dd);
      int c = 0;
      if (ts >= 0) {
        c = A.ring_cnt[(int)(ts % A.R)];
        c = c < A.cap ? c : A.cap;
      }
      s_pref[dd + 1] = c;
      local += c;
    }
  }
  int excl;
  Scan(scan_tmp).ExclusiveSum(local, excl);
  __syncthreads();
  for (int j = 0; j < per; j++) {
    int dd = b0 + j;
    if (dd < dspan) {
      excl += s_pref[dd + 1];
      s_pref[dd + 1] = excl;
    }
  }
  if (threadIdx.x == 0) s_pref[0] = 0;
  __syncthreads();
  const int total = s_pref[dspan];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // slot tidx+1 was last read two steps ago (R >= dmax + 3): reset for the next step
    A.ring_cnt[(int)((tidx + 1) % A.R)] = 0;
    clk->pending = 1;
  }
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * DELIVER_THREADS + threadIdx.x) >> 5;
  const int nwarp = (gridDim.x * DELIVER_THREADS) >> 5;
  unsigned long long nev = 0;
  for (int item = warp; item < total; item += nwarp) {
    int lo = 0, hi = dspan;   // find dd with s_pref[dd] <= item < s_pref[dd+1]
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (s_pref[mid] <= item) lo = mid; else hi = mid;
    }
    const int dd = lo;
    const int j = item - s_pref[dd];
    const long long ts = tidx - 1 - (A.dmin + dd);
    const int2 sp = A.ring[(size_t)(ts % A.R) * A.cap + j];
    const float height = __int_as_float(sp.y);
    const size_t key = (size_t)sp.x * dspan + dd;
    const long long e0 = A.ev_off[key], e1 = A.ev_off[key + 1];
    for (long long e = e0 + lane; e < e1; e += 32) {
      const EdgeW ew = A.edge[e];
      atomicAdd(&A.acc[ew.acc], (double)__fmul_rn(height, ew.w));
    }
    nev += (unsigned long long)(e1 - e0);
  }
  if (lane == 0 && nev) atomicAdd(A.n_events, nev);
}

// ---------------------------------------------------------------------------
// Records (src/multimeter.cu:76-110): one row per step into a device buffer.
// ---------------------------------------------------------------------------
__global__ void record_kernel(const RecCol *cols, int ncol, float *buf, const int *last_tidx,
                              const float *last_height, const unsigned char *has_out, Clock *clk,
                              int k, float dt) {
  long long it, tidx;
  double tnow;
  step_time(clk, k, dt, it, tidx, tnow);
  const long long row = it - clk->rec_it0;
  float *r = buf + (size_t)row * (ncol + 1);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) r[0] = (float)tnow;
  if (c < ncol) {
    RecCol rc = cols[c];
    float v;
    if (rc.ptr) v = *rc.ptr;
    else v = (has_out[rc.node] && last_tidx[rc.node] == (int)tidx) ? last_height[rc.node] : 0.0f;
    r[c + 1] = v;
  }
}

__global__ void clock_advance_kernel(Clock *clk, int K) { clk->it0 += K; }

__global__ void clock_clear_pending_kernel(Clock *clk) { clk->pending = 0; }

// ---------------------------------------------------------------------------
// Generic-port aeif kernel
// ---------------------------------------------------------------------------
template <int MODEL>
__device__ __forceinline__ void aeif_derivs_gen(const float *y, float *dy, const float *sp,
                                                const float *E_rev, const float *it1,
                                                const float *it2, int P, float refr) {
  typedef AeifShape<MODEL> S;
  const float V = (refr > 0.0f) ? sp[AP_V_reset] : ((y[0] < sp[AP_V_peak]) ? y[0] : sp[AP_V_peak]);
  const float w = y[1];
  float I = 0.0f;
  for (int i = 0; i < P; i++) {
    if (S::cond) I = __fmaf_rn(y[2 + 2 * i], __fsub_rn(E_rev[i], V), I);
    else I = __fadd_rn(I, y[2 + S::npv * i]);
  }
  float Vs;
  if (!S::cond && sp[AP_Delta_T] == 0.0f) Vs = 0.0f;
  else Vs = __fmul_rn(sp[AP_Delta_T], exp_m(__fmul_rn(__fsub_rn(V, sp[AP_V_th]), sp[AP_inv_Delta_T])));
  float s = __fmaf_rn(-sp[AP_g_L], __fsub_rn(__fsub_rn(V, sp[AP_E_L]), Vs), I);
  s = __fsub_rn(s, w);
  s = __fadd_rn(s, sp[AP_I_e]);
  dy[0] = (refr > 0.0f) ? 0.0f : __fmul_rn(s, sp[AP_inv_C_m]);
  dy[1] = __fmul_rn(__fmaf_rn(sp[AP_a], __fsub_rn(V, sp[AP_E_L]), -w), sp[AP_inv_tau_w]);
  for (int i = 0; i < P; i++) {
    if (MODEL == M_AEIF_PSC_EXP) {
      dy[2 + i] = __fmul_rn(-y[2 + i], it1[i]);
    } else {
      dy[3 + 2 * i] = __fmul_rn(-y[3 + 2 * i], it1[i]);
      dy[2 + 2 * i] = __fmaf_rn(-y[2 + 2 * i], it2[i], y[3 + 2 * i]);
    }
  }
}

template <int MODEL, bool FLUSH>
__global__ void __launch_bounds__(128) aeif_update_kernel_gen(const AeifArgs A, const SpikeOut so,
                                                              Clock *clk, int k) {
  typedef AeifShape<MODEL> S;
  constexpr int NVM = 2 + 2 * MAX_PORT;
  const StepT t = step_times<FLUSH>(clk, k, A.dt);
  const long long tidx = t.tidx;
  const double tnow = t.tnow;
  const bool pending = clk->pending != 0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nd = 0;
  if (i < A.n) {
    const int n = A.n, P = A.nport, NV = A.nvar;
    float sp[AEIF_NSCAL], E_rev[MAX_PORT], it1[MAX_PORT], it2[MAX_PORT], pw[MAX_PORT];
    for (int j = 0; j < AEIF_NSCAL; j++) sp[j] = pget(A, j, i);
    for (int p = 0; p < P; p++) {
      const int b = AEIF_NSCAL + AEIF_NPORTPAR * p;
      E_rev[p] = pget(A, b, i);
      it1[p] = pget(A, b + 1, i);
      it2[p] = pget(A, b + 2, i);
      pw[p] = pget(A, b + 3, i);
    }
    float y[NVM];
    for (int v = 0; v < NV; v++) y[v] = A.var[(size_t)v * n + i];
    if (pending) {
      double in[MAX_PORT];
      gather_inputs(in, P, n, i, A.acc, A.pin_off, A.pin, A.gen, A.lam_scale, A.seed, t.tidx_prev,
                    t.t_prev);
      for (int p = 0; p < P; p++) {
        if (in[p] != 0.0) {
          const int iv = 2 + S::npv * p + S::in_var;
          y[iv] = (float)__fma_rn(in[p], (double)pw[p], (double)y[iv]);
          if (FLUSH) A.var[(size_t)iv * n + i] = y[iv];
        }
      }
    }
    if (!FLUSH) {
      float refr = A.refr[i];
      double x = A.x[i];
      float h = A.h[i];
      const double x1 = tnow;
      bool end = false;
      int guard = 0;
      while (!end) {
        float hmax = (float)(x1 - x);
        // --- RK5 step with runtime port count
        float k1[NVM], k2[NVM], k3[NVM], k4[NVM], k5[NVM], k6[NVM], yn[NVM], iys[NVM];
        aeif_derivs_gen<MODEL>(y, k1, sp, E_rev, it1, it2, P, refr);
        for (int v = 0; v < NV; v++) {
          float ys = __fadd_rn(__fadd_rn(fabsf(y[v]), fabsf(__fmul_rn(k1[v], h))), ck::scal_min);
          iys[v] = __fdiv_rn(1.0f, ys);
        }
        int trials = 0;
        float err;
        nd += 1;
        for (;;) {
          if (h > hmax) h = hmax;
          if (h < A.hmin) h = A.hmin;
          const float b21 = __fmul_rn(h, ck::a21), b31 = __fmul_rn(h, ck::a31), b32 = __fmul_rn(h, ck::a32),
                      b41 = __fmul_rn(h, ck::a41), b42 = __fmul_rn(h, ck::a42), b43 = __fmul_rn(h, ck::a43),
                      b51 = __fmul_rn(h, ck::a51), b52 = __fmul_rn(h, ck::a52), b53 = __fmul_rn(h, ck::a53),
                      b54 = __fmul_rn(h, ck::a54), b61 = __fmul_rn(h, ck::a61), b62 = __fmul_rn(h, ck::a62),
                      b63 = __fmul_rn(h, ck::a63), b64 = __fmul_rn(h, ck::a64), b65 = __fmul_rn(h, ck::a65),
                      b71 = __fmul_rn(h, ck::a71), b73 = __fmul_rn(h, ck::a73), b74 = __fmul_rn(h, ck::a74),
                      b76 = __fmul_rn(h, ck::a76), f1 = __fmul_rn(h, ck::e1), f3 = __fmul_rn(h, ck::e3),
                      f4 = __fmul_rn(h, ck::e4), f5 = __fmul_rn(h, ck::e5), f6 = __fmul_rn(h, ck::e6);
          for (int v = 0; v < NV; v++) yn[v] = __fmaf_rn(b21, k1[v], y[v]);
          aeif_derivs_gen<MODEL>(yn, k2, sp, E_rev, it1, it2, P, refr);
          for (int v = 0; v < NV; v++) yn[v] = __fmaf_rn(b32, k2[v], __fmaf_rn(b31, k1[v], y[v]));
          aeif_derivs_gen<MODEL>(yn, k3, sp, E_rev, it1, it2, P, refr);
          for (int v = 0; v < NV; v++)
            yn[v] = __fmaf_rn(b43, k3[v], __fmaf_rn(b42, k2[v], __fmaf_rn(b41, k1[v], y[v])));
          aeif_derivs_gen<MODEL>(yn, k4, sp, E_rev, it1, it2, P, refr);
          for (int v = 0; v < NV; v++)
            yn[v] = __fmaf_rn(b54, k4[v], __fmaf_rn(b53, k3[v], __fmaf_rn(b52, k2[v], __fmaf_rn(b51, k1[v], y[v]))));
          aeif_derivs_gen<MODEL>(yn, k5, sp, E_rev, it1, it2, P, refr);
          for (int v = 0; v < NV; v++)
            yn[v] = __fmaf_rn(b65, k5[v], __fmaf_rn(b64, k4[v], __fmaf_rn(b63, k3[v],
                              __fmaf_rn(b62, k2[v], __fmaf_rn(b61, k1[v], y[v])))));
          aeif_derivs_gen<MODEL>(yn, k6, sp, E_rev, it1, it2, P, refr);
          for (int v = 0; v < NV; v++)
            yn[v] = __fmaf_rn(b76, k6[v], __fmaf_rn(b74, k4[v], __fmaf_rn(b73, k3[v], __fmaf_rn(b71, k1[v], y[v]))));
          err = 0.0f;
          for (int v = 0; v < NV; v++) {
            float e = __fmaf_rn(f6, k6[v], __fmaf_rn(f5, k5[v], __fmaf_rn(f4, k4[v],
                                __fmaf_rn(f3, k3[v], __fmul_rn(f1, k1[v])))));
            float av = fabsf(__fmul_rn(e, iys[v]));
            err = (err > av) ? err : av;
          }
          err = __fmul_rn(err, ck::inv_eps);
          nd += 5;
          trials++;
          if (err <= 1.0f || h <= A.hmin_acc) break;
          if (trials >= ck::max_trials) {
            atomicOr(so.status, ST_RK5_TRIALS);
            break;
          }
          float hnew = __fmul_rn(__fmul_rn(h, ck::coeff), __fdiv_rn(1.0f, __fsqrt_rn(__fsqrt_rn(err))));
          float h01 = __fmul_rn(0.1f, h);
          h = (hnew > h01) ? hnew : h01;
        }
        x += (double)h;
        if (err > ck::err_min) h = __fmul_rn(__fmul_rn(h, ck::coeff), exp_m(__fmul_rn(-0.2f, log_m(err))));
        else h = __fmul_rn(5.0f, h);
        if (!(h == h)) h = A.hmin;
        for (int v = 0; v < NV; v++) y[v] = yn[v];
        // --- end of step
        end = (x >= x1 - (double)A.hmin);
        if (++guard > ck::max_substeps) {
          atomicOr(so.status, ST_RK5_TRIALS);
          break;
        }
        if (y[0] < -1.0e3f) {
          y[0] = sp[AP_V_reset];
          y[1] = 0.0f;
          atomicOr(so.status, ST_NUMERIC);
          continue;
        }
        if (y[1] < -1.0e6f || y[1] > 1.0e6f) {
          y[0] = sp[AP_V_reset];
          y[1] = 0.0f;
          atomicOr(so.status, ST_NUMERIC);
          continue;
        }
        if (refr > 0.0f) {
          y[0] = sp[AP_V_reset];
          if (end) refr = __fsub_rn(refr, 1.0f);
        } else if (y[0] >= sp[AP_V_peak]) {
          push_spike(so, A.rec, A.i0 + i, i, 1.0f, tidx, tnow);
          y[0] = sp[AP_V_reset];
          y[1] = __fadd_rn(y[1], sp[AP_b]);
          refr = sp[AP_refr_steps];
        }
      }
      for (int v = 0; v < NV; v++) A.var[(size_t)v * n + i] = y[v];
      A.refr[i] = refr;
      A.x[i] = x;
      A.h[i] = h;
    }
  }
  if (!FLUSH) {
    for (int o = 16; o > 0; o >>= 1) nd += __shfl_down_sync(0xffffffffu, nd, o);
    if ((threadIdx.x & 31) == 0 && nd) atomicAdd(A.nderiv, nd);
  }
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
template <int MODEL, bool FLUSH>
static int launch_aeif_model(const AeifArgs &A, const SpikeOut &so, Clock *clk, int k,
                             cudaStream_t st) {
  dim3 grid((A.n + 127) / 128), block(128);
  dim3 sgrid(std::min((A.n + 127) / 128, 148 * 2));
  const bool strag = !FLUSH && A.budget > 0;
  switch (A.nport) {
  case 1:
    aeif_update_kernel<MODEL, 1, FLUSH><<<grid, block, 0, st>>>(A, so, clk, k);
    if (strag) aeif_straggler_kernel<MODEL, 1><<<sgrid, block, 0, st>>>(A, so, clk, k);
    break;
  case 2:
    aeif_update_kernel<MODEL, 2, FLUSH><<<grid, block, 0, st>>>(A, so, clk, k);
    if (strag) aeif_straggler_kernel<MODEL, 2><<<sgrid, block, 0, st>>>(A, so, clk, k);
    break;
  case 3:
    aeif_update_kernel<MODEL, 3, FLUSH><<<grid, block, 0, st>>>(A, so, clk, k);
    if (strag) aeif_straggler_kernel<MODEL, 3><<<sgrid, block, 0, st>>>(A, so, clk, k);
    break;
  case 4:
    aeif_update_kernel<MODEL, 4, FLUSH><<<grid, block, 0, st>>>(A, so, clk, k);
    if (strag) aeif_straggler_kernel<MODEL, 4><<<sgrid, block, 0, st>>>(A, so, clk, k);
    break;
  default:
    aeif_update_kernel_gen<MODEL, FLUSH><<<grid, block, 0, st>>>(A, so, clk, k);
    return 1;
  }
  return strag ? 2 : 1;
}

// Returns the number of kernels launched.
int launch_aeif(int model, bool flush, const AeifArgs &A, const SpikeOut &so, Clock *clk, int k,
                cudaStream_t st) {
  if (A.n <= 0) return 0;
  if (flush) {
    switch (model) {
    case M_AEIF_COND_BETA: return launch_aeif_model<M_AEIF_COND_BETA, true>(A, so, clk, k, st);
    case M_AEIF_COND_ALPHA: return launch_aeif_model<M_AEIF_COND_ALPHA, true>(A, so, clk, k, st);
    case M_AEIF_PSC_EXP: return launch_aeif_model<M_AEIF_PSC_EXP, true>(A, so, clk, k, st);
    case M_AEIF_PSC_ALPHA: return launch_aeif_model<M_AEIF_PSC_ALPHA, true>(A, so, clk, k, st);
    }
  } else {
    switch (model) {
    case M_AEIF_COND_BETA: return launch_aeif_model<M_AEIF_COND_BETA, false>(A, so, clk, k, st);
    case M_AEIF_COND_ALPHA: return launch_aeif_model<M_AEIF_COND_ALPHA, false>(A, so, clk, k, st);
    case M_AEIF_PSC_EXP: return launch_aeif_model<M_AEIF_PSC_EXP, false>(A, so, clk, k, st);
    case M_AEIF_PSC_ALPHA: return launch_aeif_model<M_AEIF_PSC_ALPHA, false>(A, so, clk, k, st);
    }
  }
  return 0;
}

void launch_iaf(bool flush, const IafArgs &A, const SpikeOut &so, Clock *clk, int k, float dt,
                cudaStream_t st) {
  if (A.n <= 0) return;
  dim3 grid((A.n + 255) / 256), block(256);
  if (flush) iaf_update_kernel<true><<<grid, block, 0, st>>>(A, so, clk, k, dt);
  else iaf_update_kernel<false><<<grid, block, 0, st>>>(A, so, clk, k, dt);
}

void launch_spike_gen(const SpikeGenArgs &A, const SpikeOut &so, Clock *clk, int k, float dt,
                      cudaStream_t st) {
  if (A.n <= 0) return;
  spike_gen_kernel<<<(A.n + 255) / 256, 256, 0, st>>>(A, so, clk, k, dt);
}

void launch_deliver(const DeliverArgs &A, int n_blocks, Clock *clk, int k, float dt, cudaStream_t st) {
  size_t smem = (size_t)(A.dspan + 1) * sizeof(int);
  deliver_kernel<<<n_blocks, DELIVER_THREADS, smem, st>>>(A, clk, k, dt);
}

void launch_record(const RecCol *cols, int ncol, float *buf, const int *last_tidx,
                   const float *last_height, const unsigned char *has_out, Clock *clk, int k,
                   float dt, cudaStream_t st) {
  int nb = (ncol + 127) / 128;
  if (nb < 1) nb = 1;
  record_kernel<<<nb, 128, 0, st>>>(cols, ncol, buf, last_tidx, last_height, has_out, clk, k, dt);
}

void launch_clock_advance(Clock *clk, int K, cudaStream_t st) {
  clock_advance_kernel<<<1, 1, 0, st>>>(clk, K);
}

void launch_clock_clear_pending(Clock *clk, cudaStream_t st) {
  clock_clear_pending_kernel<<<1, 1, 0, st>>>(clk);
}

int deliver_max_dspan() { return MAX_DSPAN; }

}  // namespace ngpu
