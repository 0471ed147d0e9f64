// Device code of the aeif_*_multisynapse update shared by the plain kernels
// (ngpu_kernels.cu) and the learned-step-size variants (ngpu_learn.cu): the
// Cash-Karp RK5 step, the sub-step loop with the model's ExternalUpdate, the
// end-of-step record and input fold, and the batch / straggler kernels.
//
// LM (learn mode) selects what a step does besides the reference algorithm:
//   LM_PLAIN   the reference step-size controller alone;
//   LM_LOG     additionally appends one tuple (step features, accepted h, error)
//              per accepted step to a device log;
//   LM_PROPOSE a small MLP proposes the first trial h of a step whenever the plain
//              controller's h would not reach the end of the time step; the error
//              test, the rejection shrink and the controller update are unchanged.
#pragma once
#include "ngpu_math.cuh"
#include "ngpu_stepmodel.h"
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

// Programmatic dependent launch. A kernel launched with programmatic stream serialization
// may be scheduled while its predecessor in the stream still runs. Every kernel of the step
// loop therefore first waits until its predecessor grid has completed and its memory is
// visible, and only then lets its own successor be scheduled; before the wait it touches no
// global memory. So the order of memory effects is that of plain stream order, and what
// overlaps is the launch and block scheduling of the next kernel. Without the launch
// attribute both instructions do nothing.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Set by the engine around the launches of one time batch (ngpu_kernels.cu).
extern bool g_launch_pdl;

// kern<<<grid, block, smem, st>>>(args...), with programmatic stream serialization when
// g_launch_pdl is set.
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args... args) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = g_launch_pdl ? at : nullptr;
  cfg.numAttrs = g_launch_pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

// Step `m` of the batch starting at graph step k0.
struct StepT {
  long long it, tidx;
  double tnow;
};

// The clock is read once per kernel (it changes only between graphs) and passed by value,
// so the per-step time needs no memory access.
__device__ __forceinline__ StepT step_at(const Clock &c, int k0, int m, float dt) {
  StepT s;
  s.it = c.it0 + k0 + m;
  s.tidx = c.tidx_base + s.it + 1;
  s.tnow = c.t0 + (double)dt * (double)(s.it + 1);
  return s;
}

// PushSpike (src/spike_buffer.cu:162-242) on the ring design.  RING = false (delivery at
// emission): the spike goes to no ring, its out-edges are added by the caller.
template <bool RING = true>
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
  if (so.last_rev) {
    // the spike reaches the node's own synapses (STDP) now or den_delay steps later
    // (src/spike_buffer.cu:183-186, 279-281, 314-316)
    const int D = so.den_steps ? so.den_steps[node] : 0;
    if (D == 0) {
      so.last_rev[node] = (int)tidx;
    } else {
      const int rs = (int)((tidx + D) % so.rev_R);
      const int pos = atomicAdd(&so.rev_cnt[rs], 1);
      if (pos < so.rev_cap) so.rev_ring[(size_t)rs * so.rev_cap + pos] = node;
      else atomicOr(so.status, ST_RING_OVERFLOW);
    }
  }
  if (so.xch && so.has_out_all[node]) {
    // partitioned network: other processes may deliver this spike
    const int pos = atomicAdd(&so.xch[0].x, 1);
    if (pos < so.xch_cap) so.xch[1 + pos] = make_int4(node, __float_as_int(height), (int)tidx, 0);
    else atomicOr(so.status, ST_EXCHANGE_FULL);
  }
  if (RING && so.has_out[node]) {
    int slot = (int)(tidx % so.R);
    int pos = atomicAdd(&so.ring_cnt[slot], 1);
    if (pos < so.cap) so.ring[(size_t)slot * so.cap + pos] = make_int2(node, __float_as_int(height));
    else atomicOr(so.status, ST_RING_OVERFLOW);
  }
}

// The poiss_gen edges of a neuron do not change during a batch: with exactly one edge
// (the common case) it, its generator, the mean count lam and exp(-lam) are loaded once
// per batch, and the edge's current Philox block (four steps) is kept across steps.
struct PoissonCache {
  int e0, e1;
  PoissonIn pe;
  GenPar g;
  float lam, emlam;
  long long blk;
  U4 r;
};

// The edge tables and the generator table change only between kernels (calibration, host
// copies between Simulate calls): they are read through the read-only data path.
__device__ __forceinline__ PoissonIn ldg_pin(const PoissonIn *p) {
  static_assert(sizeof(PoissonIn) == 24, "PoissonIn is three 8-byte words");
  const uint2 *q = reinterpret_cast<const uint2 *>(p);
  const uint2 a = __ldg(q), b = __ldg(q + 1), d = __ldg(q + 2);
  PoissonIn e;
  e.edge_id = a.x;
  e.gen = (int)a.y;
  e.weight = __uint_as_float(b.x);
  e.delay = __uint_as_float(b.y);
  e.port = (int)d.x;
  e.stream = d.y;
  return e;
}

// 64-bit Philox counter key of a poiss_gen edge: (generator stream, out-edge index).
__device__ __forceinline__ uint64_t pin_key(const PoissonIn &pe) {
  return ((uint64_t)pe.stream << 32) | (uint64_t)pe.edge_id;
}

__device__ __forceinline__ GenPar ldg_gen(const GenPar *p) {
  static_assert(sizeof(GenPar) == 16, "GenPar is one 16-byte word");
  const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
  GenPar g;
  g.rate = v.x;
  g.origin = v.y;
  g.start = v.z;
  g.stop = v.w;
  return g;
}

__device__ __forceinline__ void poisson_cache_load(const GroupInput &G, int i, PoissonCache &c) {
  c.e0 = c.e1 = 0;
  c.blk = -1;
  if (G.pin_off) {
    c.e0 = __ldg(G.pin_off + i);
    c.e1 = __ldg(G.pin_off + i + 1);
    if (c.e1 - c.e0 == 1) {
      c.pe = ldg_pin(G.pin + c.e0);
      c.g = ldg_gen(G.gen + c.pe.gen);
      c.lam = __fmul_rn(G.lam_scale, c.g.rate);
      c.emlam = exp_m(-c.lam);
    }
  }
}

// in[port] += v with the port known only at run time, written as a compare per port so
// that `in` stays in registers (an indexed store would place it in local memory).
template <int PMAX>
__device__ __forceinline__ void add_to_port(double *in, int port, double v) {
#pragma unroll
  for (int p = 0; p < PMAX; p++)
    if (p == port) in[p] += v;
}

// The cached edge's draw: the same value as poisson_draw, without recomputing exp(-lam)
// and with one Philox call per four steps.
template <int PMAX>
__device__ __forceinline__ void poisson_add_cached(double *in, const GroupInput &G, PoissonCache &c, long long tidx,
                                                   double tnow) {
  const double t_rel = tnow - (double)c.g.origin - (double)c.pe.delay;
  if (t_rel >= (double)c.g.start && t_rel <= (double)c.g.stop) {
    int k;
    if (c.lam > 0.0f && c.lam <= 10.0f) {
      const long long b = tidx >> 2;
      if (b != c.blk) {
        c.r = poisson_block(G.seed, pin_key(c.pe), tidx, 0);
        c.blk = b;
      }
      k = poisson_small(c.lam, c.emlam, u01(word_of(c.r, (int)(tidx & 3))));
    } else {
      k = poisson_draw(c.lam, G.seed, pin_key(c.pe), tidx);
    }
    if (k > 0) add_to_port<PMAX>(in, c.pe.port, (double)__fmul_rn(c.pe.weight, (float)k));
  }
}

template <int PMAX>
__device__ __forceinline__ void poisson_add(double *in, const GroupInput &G, const PoissonIn &pe, const GenPar &g,
                                            long long tidx, double tnow) {
  const double t_rel = tnow - (double)g.origin - (double)pe.delay;
  if (t_rel >= (double)g.start && t_rel <= (double)g.stop) {
    int k = poisson_draw(__fmul_rn(G.lam_scale, g.rate), G.seed, pin_key(pe), tidx);
    if (k > 0) add_to_port<PMAX>(in, pe.port, (double)__fmul_rn(pe.weight, (float)k));
  }
}

// Spike input of step m, read at the start of the step so that the load latency hides
// behind the step's integration (the delivery of the batch finished before the kernel).
template <int PMAX>
__device__ __forceinline__ void acc_prefetch(double *a, int np, int n, int i, const GroupInput &G, int m) {
  const double *acc = G.acc + (size_t)m * G.slot_stride;
#pragma unroll
  for (int p = 0; p < PMAX; p++) a[p] = (p < np) ? acc[(size_t)p * n + i] : 0.0;
}

// Input arriving in step (tidx, tnow) for neuron i: the accumulator slot m (spikes
// delivered this step, src/get_spike.cu:60-108), prefetched, plus this step's poiss_gen
// draws (src/poiss_gen.cu:55-86); the nonzero accumulator entries are cleared for their
// next use.
template <int PMAX>
__device__ __forceinline__ void step_inputs_pf(double *in, const double *a, int np, int n, int i,
                                               const GroupInput &G, PoissonCache &c, int m, long long tidx,
                                               double tnow) {
  double *acc = G.acc + (size_t)m * G.slot_stride;
#pragma unroll
  for (int p = 0; p < PMAX; p++) {
    in[p] = a[p];
    if (p < np && a[p] != 0.0) acc[(size_t)p * n + i] = 0.0;
  }
  if (c.e1 - c.e0 == 1) {
    poisson_add_cached<PMAX>(in, G, c, tidx, tnow);
  } else {
    for (int e = c.e0; e < c.e1; e++) {
      const PoissonIn pe = G.pin[e];
      poisson_add<PMAX>(in, G, pe, G.gen[pe.gen], tidx, tnow);
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

// PMAX: compile-time bound on the port count; FIXED: the group has exactly PMAX ports.
template <int MODEL, int PMAX, bool FIXED> struct AeifQ {
  int np;
  float V_th, Delta_T, inv_Delta_T, g_L, E_L, inv_C_m, a, b, inv_tau_w, I_e, V_peak, V_reset,
      refr_steps;
  float E_rev[PMAX], inv_t1[PMAX], inv_t2[PMAX], pw[PMAX];
  __device__ __forceinline__ int ports() const { return FIXED ? PMAX : np; }
};

template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ void aeif_derivs(const float *y, float *dy,
                                            const AeifQ<MODEL, PMAX, FIXED> &q, float refr) {
  typedef AeifShape<MODEL> S;
  const int np = q.ports();
  const float V = (refr > 0.0f) ? q.V_reset : ((y[0] < q.V_peak) ? y[0] : q.V_peak);
  const float w = y[1];
  float I = 0.0f;
#pragma unroll
  for (int i = 0; i < PMAX; i++) {
    if (i < np) {
      if (S::cond) I = __fmaf_rn(y[2 + 2 * i], __fsub_rn(q.E_rev[i], V), I);
      else I = __fadd_rn(I, y[2 + S::npv * i]);
    }
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
  for (int i = 0; i < PMAX; i++) {
    if (i < np) {
      if (MODEL == M_AEIF_PSC_EXP) {
        dy[2 + i] = __fmul_rn(-y[2 + i], q.inv_t1[i]);
      } else {
        dy[3 + 2 * i] = __fmul_rn(-y[3 + 2 * i], q.inv_t1[i]);
        dy[2 + 2 * i] = __fmaf_rn(-y[2 + 2 * i], q.inv_t2[i], y[3 + 2 * i]);
      }
    }
  }
}

// UNI: every parameter of the group is uniform, so each one is read from the kernel
// arguments (constant bank) where it is used and needs no register of its own.
template <bool UNI = false>
__device__ __forceinline__ float pget(const AeifArgs &A, int j, int i) {
  if (UNI) return A.pval[j];
  const float *p = A.parr[j];
  return p ? __ldg(p + i) : A.pval[j];
}

template <int MODEL, int PMAX, bool FIXED, bool UNI = false>
__device__ __forceinline__ void load_aeif_par(const AeifArgs &A, int i, AeifQ<MODEL, PMAX, FIXED> &q) {
  q.np = A.nport;
  q.V_th = pget<UNI>(A, AP_V_th, i);
  q.Delta_T = pget<UNI>(A, AP_Delta_T, i);
  q.inv_Delta_T = pget<UNI>(A, AP_inv_Delta_T, i);
  q.g_L = pget<UNI>(A, AP_g_L, i);
  q.E_L = pget<UNI>(A, AP_E_L, i);
  q.inv_C_m = pget<UNI>(A, AP_inv_C_m, i);
  q.a = pget<UNI>(A, AP_a, i);
  q.b = pget<UNI>(A, AP_b, i);
  q.inv_tau_w = pget<UNI>(A, AP_inv_tau_w, i);
  q.I_e = pget<UNI>(A, AP_I_e, i);
  q.V_peak = pget<UNI>(A, AP_V_peak, i);
  q.V_reset = pget<UNI>(A, AP_V_reset, i);
  q.refr_steps = pget<UNI>(A, AP_refr_steps, i);
  const int np = q.ports();
#pragma unroll
  for (int p = 0; p < PMAX; p++) {
    if (p < np) {
      const int b = AEIF_NSCAL + AEIF_NPORTPAR * p;
      q.E_rev[p] = pget<UNI>(A, b + 0, i);
      q.inv_t1[p] = pget<UNI>(A, b + 1, i);
      q.inv_t2[p] = pget<UNI>(A, b + 2, i);
      q.pw[p] = pget<UNI>(A, b + 3, i);
    }
  }
}

// sign(x) log(1 + |x|): derivatives span many decades (dV/dt near the spike peak).
__device__ __forceinline__ float slog(float x) {
  const float l = log_m(__fadd_rn(1.0f, fabsf(x)));
  return (x < 0.0f) ? -l : l;
}

// Features of a step for the learned proposal (definition in ngpu_stepmodel.h).
template <int MODEL, int PMAX>
__device__ __forceinline__ void step_features(const float *y, const float *k1, int np, float h_in,
                                              float hmax, float *f) {
  typedef AeifShape<MODEL> S;
  f[0] = y[0];
  f[1] = y[1];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    float v = 0.0f;
    if (p < PMAX && p < np) v = y[2 + S::npv * (p < PMAX ? p : 0)];
    f[2 + p] = v;
  }
  float s = 0.0f;
#pragma unroll
  for (int p = 0; p < PMAX; p++)
    if (p < np) s = __fadd_rn(s, k1[2 + S::npv * p]);
  f[6] = slog(k1[0]);
  f[7] = slog(s);
  f[8] = log_m(h_in);
  f[9] = log_m(hmax);
}

// MLP output for features f; M is the flat parameter vector (in shared memory).
__device__ __forceinline__ float mlp_out(const float *M, const float *f) {
  float xn[SM_NF];
#pragma unroll
  for (int k = 0; k < SM_NF; k++) {
    const float v = __fmul_rn(__fsub_rn(f[k], M[SM_MU + k]), M[SM_ISIG + k]);
    xn[k] = fminf(fmaxf(v, -SM_XCLAMP), SM_XCLAMP);
  }
  float a1[SM_NH];
#pragma unroll
  for (int j = 0; j < SM_NH; j++) {
    float z = M[SM_B1 + j];
#pragma unroll
    for (int k = 0; k < SM_NF; k++) z = __fmaf_rn(M[SM_W1 + j * SM_NF + k], xn[k], z);
    a1[j] = (z > 0.0f) ? z : 0.0f;
  }
  float out = M[SM_B3];
#pragma unroll 4
  for (int j = 0; j < SM_NH; j++) {
    float z = M[SM_B2 + j];
#pragma unroll
    for (int k = 0; k < SM_NH; k++) z = __fmaf_rn(M[SM_W2 + j * SM_NH + k], a1[k], z);
    z = (z > 0.0f) ? z : 0.0f;
    out = __fmaf_rn(M[SM_W3 + j], z, out);
  }
  return out;
}

// Proposed step size: safety * exp(out * label_sigma + label_mu).
__device__ __forceinline__ float mlp_propose(const float *M, const float *f) {
  const float o = mlp_out(M, f);
  return __fmul_rn(M[SM_SAFETY], exp_m(__fmaf_rn(o, M[SM_LSIG], M[SM_LMU])));
}

// Stage combination r[i] = y[i] + b1 k1[i] + ... + bK kK[i] as the FMA chain innermost-first,
// two state variables per instruction with sm_100's packed FP32 FMA. Each lane of __ffma2_rn
// is rounded exactly as the scalar __fmaf_rn, so r is bit for bit the scalar chain's. A pair
// whose upper variable lies past NV (odd variable count) computes an unused upper lane.
// PAIR = false keeps one variable per instruction (the groups with a runtime port count, whose
// arrays do not fit in registers either way).
template <int NVM, int K, bool PAIR>
__device__ __forceinline__ void stage_comb(float *r, const float *y, int NV, const float *k1, float b1,
                                           const float *k2 = nullptr, float b2 = 0.0f,
                                           const float *k3 = nullptr, float b3 = 0.0f,
                                           const float *k4 = nullptr, float b4 = 0.0f,
                                           const float *k5 = nullptr, float b5 = 0.0f) {
#pragma unroll
  for (int i = 0; i < NVM; i += (PAIR ? 2 : 1)) {
    if (i < NV) {
      if (PAIR && i + 1 < NVM) {
        float2 a = __ffma2_rn(make_float2(b1, b1), make_float2(k1[i], k1[i + 1]), make_float2(y[i], y[i + 1]));
        if (K > 1) a = __ffma2_rn(make_float2(b2, b2), make_float2(k2[i], k2[i + 1]), a);
        if (K > 2) a = __ffma2_rn(make_float2(b3, b3), make_float2(k3[i], k3[i + 1]), a);
        if (K > 3) a = __ffma2_rn(make_float2(b4, b4), make_float2(k4[i], k4[i + 1]), a);
        if (K > 4) a = __ffma2_rn(make_float2(b5, b5), make_float2(k5[i], k5[i + 1]), a);
        r[i] = a.x;
        r[i + 1] = a.y;
      } else {
        float a = __fmaf_rn(b1, k1[i], y[i]);
        if (K > 1) a = __fmaf_rn(b2, k2[i], a);
        if (K > 2) a = __fmaf_rn(b3, k3[i], a);
        if (K > 3) a = __fmaf_rn(b4, k4[i], a);
        if (K > 4) a = __fmaf_rn(b5, k5[i], a);
        r[i] = a;
      }
    }
  }
}

// The pieces of one RK5 step (src/rk5.h:69-159), shared by the step-at-once form
// (rk5_step) and the trial-per-iteration form of the plain batch kernel.
//
// rk5_begin: k1 = f(y) and the reciprocal error scale 1 / (|y| + |h k1| + scal_min), with the
// h entering the step (the reference computes y_scal before clamping h).
template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ void rk5_begin(const float *y, float h, const AeifQ<MODEL, PMAX, FIXED> &q, float refr,
                                          float *k1, float *iys) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
  const int NV = 2 + AeifShape<MODEL>::npv * q.ports();
  aeif_derivs(y, k1, q, refr);
#pragma unroll
  for (int i = 0; i < NVM; i++) {
    if (i < NV) {
      float ys = __fadd_rn(__fadd_rn(fabsf(y[i]), fabsf(__fmul_rn(k1[i], h))), ck::scal_min);
      iys[i] = __fdiv_rn(1.0f, ys);
    }
  }
}

// rk5_trial: one trial with h clamped to [hmin, hmax] (h keeps the clamped value): the
// 5th-order solution in yn and the scaled error estimate (accept when <= 1).  Five
// derivative evaluations.
template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ float rk5_trial(const float *y, float &h, float hmin, float hmax,
                                           const AeifQ<MODEL, PMAX, FIXED> &q, float refr, const float *k1,
                                           const float *iys, float *yn) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
  const int NV = 2 + AeifShape<MODEL>::npv * q.ports();
  float k2[NVM], k3[NVM], k4[NVM], k5[NVM], k6[NVM];
  if (h > hmax) h = hmax;
  if (h < hmin) h = hmin;
  // each stage's coefficients h * a_ij are formed just before the stage (short live ranges)
  stage_comb<NVM, 1, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a21));
  aeif_derivs(yn, k2, q, refr);
  stage_comb<NVM, 2, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a31), k2, __fmul_rn(h, ck::a32));
  aeif_derivs(yn, k3, q, refr);
  stage_comb<NVM, 3, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a41), k2, __fmul_rn(h, ck::a42), k3,
                            __fmul_rn(h, ck::a43));
  aeif_derivs(yn, k4, q, refr);
  stage_comb<NVM, 4, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a51), k2, __fmul_rn(h, ck::a52), k3,
                            __fmul_rn(h, ck::a53), k4, __fmul_rn(h, ck::a54));
  aeif_derivs(yn, k5, q, refr);
  stage_comb<NVM, 5, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a61), k2, __fmul_rn(h, ck::a62), k3,
                            __fmul_rn(h, ck::a63), k4, __fmul_rn(h, ck::a64), k5, __fmul_rn(h, ck::a65));
  aeif_derivs(yn, k6, q, refr);
  stage_comb<NVM, 4, FIXED>(yn, y, NV, k1, __fmul_rn(h, ck::a71), k3, __fmul_rn(h, ck::a73), k4,
                            __fmul_rn(h, ck::a74), k6, __fmul_rn(h, ck::a76));
  const float f1 = __fmul_rn(h, ck::e1), f3 = __fmul_rn(h, ck::e3), f4 = __fmul_rn(h, ck::e4),
              f5 = __fmul_rn(h, ck::e5), f6 = __fmul_rn(h, ck::e6);
  // error terms two variables at a time (lane-exact, as in stage_comb)
  float err = 0.0f;
#pragma unroll
  for (int i = 0; i < NVM; i += (FIXED ? 2 : 1)) {
    if (i < NV) {
      if (FIXED && i + 1 < NVM) {
        float2 v = __fmul2_rn(make_float2(f1, f1), make_float2(k1[i], k1[i + 1]));
        v = __ffma2_rn(make_float2(f3, f3), make_float2(k3[i], k3[i + 1]), v);
        v = __ffma2_rn(make_float2(f4, f4), make_float2(k4[i], k4[i + 1]), v);
        v = __ffma2_rn(make_float2(f5, f5), make_float2(k5[i], k5[i + 1]), v);
        v = __ffma2_rn(make_float2(f6, f6), make_float2(k6[i], k6[i + 1]), v);
        v = __fmul2_rn(v, make_float2(iys[i], iys[i + 1]));
        const float a0 = fabsf(v.x);
        err = (err > a0) ? err : a0;
        if (i + 1 < NV) {
          const float a1 = fabsf(v.y);
          err = (err > a1) ? err : a1;
        }
      } else {
        float v = __fmaf_rn(f6, k6[i], __fmaf_rn(f5, k5[i], __fmaf_rn(f4, k4[i],
                                                                      __fmaf_rn(f3, k3[i], __fmul_rn(f1, k1[i])))));
        float av = fabsf(__fmul_rn(v, iys[i]));
        err = (err > av) ? err : av;
      }
    }
  }
  return __fmul_rn(err, ck::inv_eps);
}

// Step size of the next trial after a rejection: max(0.9 h err^-1/4, 0.1 h).
__device__ __forceinline__ float rk5_shrink(float h, float err) {
  float hnew = __fmul_rn(__fmul_rn(h, ck::coeff), __fdiv_rn(1.0f, __fsqrt_rn(__fsqrt_rn(err))));
  float h01 = __fmul_rn(0.1f, h);
  return (hnew > h01) ? hnew : h01;
}

// Step size proposed after an accepted trial: 0.9 h err^-1/5, or 5 h for a tiny error.
__device__ __forceinline__ float rk5_grow(float h, float err, float hmin) {
  if (err > ck::err_min) h = __fmul_rn(__fmul_rn(h, ck::coeff), exp_m(__fmul_rn(-0.2f, log_m(err))));
  else h = __fmul_rn(5.0f, h);
  if (!(h == h)) h = hmin;
  return h;
}

// Largest step in [hmin, hmax] whose trial passes the error test (hmax if it passes, else a
// bisection in log h with 30 halvings): the first trial a perfect proposal would choose.
// Analysis only (LM_BOUND); its trials are not counted as evaluations.
template <int MODEL, int PMAX, bool FIXED>
__device__ __noinline__ float rk5_largest_passing(const float *y, float hmin, float hmax,
                                                  const AeifQ<MODEL, PMAX, FIXED> &q, float refr, const float *k1,
                                                  const float *iys) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
  float tmp[NVM];
  float hh = hmax;
  if (rk5_trial(y, hh, hmin, hmax, q, refr, k1, iys, tmp) <= 1.0f) return hmax;
  float lo = hmin, hi = hmax;
  for (int it = 0; it < 30; it++) {
    const float mid = (float)sqrt((double)lo * (double)hi);
    hh = mid;
    if (rk5_trial(y, hh, hmin, hmax, q, refr, k1, iys, tmp) <= 1.0f) lo = mid;
    else hi = mid;
  }
  return lo;
}

// One accepted RK5 step (src/rk5.h:69-159); returns the number of derivative evaluations.
// The error scale y_scal uses the h entering the step (the plain controller's), as in
// the reference, whatever the learned proposal chooses as the first trial.
template <int MODEL, int PMAX, bool FIXED, int LM>
__device__ __forceinline__ int rk5_step(double &x, float *y, float &h, float hmin, float hmin_acc,
                                        float hmax, const AeifQ<MODEL, PMAX, FIXED> &q, float refr,
                                        unsigned *status, const float *smodel, const LearnCtx &L) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
  const int NV = 2 + AeifShape<MODEL>::npv * q.ports();
  float k1[NVM], yn[NVM], iys[NVM];
  rk5_begin(y, h, q, refr, k1, iys);
  if constexpr (LM == LM_BOUND) h = rk5_largest_passing(y, hmin, hmax, q, refr, k1, iys);
  float f[(LM == LM_PLAIN || LM == LM_BOUND) ? 1 : SM_NF];
  if (LM == LM_LOG || (LM == LM_PROPOSE && h < hmax)) step_features<MODEL, PMAX>(y, k1, q.ports(), h, hmax, f);
  if (LM == LM_PROPOSE && h < hmax) {
    // the plain h would not reach the end of the time step: let the network propose
    const float hp = mlp_propose(smodel, f);
    if (hp > 0.0f && hp <= 3.0e38f) {        // otherwise keep the plain proposal
      const float lo = __fmul_rn(smodel[SM_FLOOR], h);
      h = (hp > lo) ? hp : lo;
    }
  }
  int nd = 1;
  int trials = 0;
  float err;
  for (;;) {
    err = rk5_trial(y, h, hmin, hmax, q, refr, k1, iys, yn);
    nd += 5;
    trials++;
    if (err <= 1.0f || h <= hmin_acc) break;
    if (trials >= ck::max_trials) {
      atomicOr(status, ST_RK5_TRIALS);
      break;
    }
    h = rk5_shrink(h, err);
  }
  if (LM == LM_LOG) {
    const unsigned long long pos = atomicAdd(L.log_cursor, 1ULL);
    if (pos < L.log_cap) {
      float *t = L.log + pos * LOG_W;
#pragma unroll
      for (int k = 0; k < SM_NF; k++) t[k] = f[k];
      t[SM_NF] = h;
      t[SM_NF + 1] = err;
    }
  }
  x += (double)h;
  h = rk5_grow(h, err, hmin);
#pragma unroll
  for (int i = 0; i < NVM; i++)
    if (i < NV) y[i] = yn[i];
  return nd;
}

template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ bool aeif_external(const AeifArgs &A, const SpikeOut &so, int i,
                                              const AeifQ<MODEL, PMAX, FIXED> &q, float *y, float &refr,
                                              double x, long long tidx, double tnow, int &guard);

// One RK5 sub-step of neuron i from x towards the end of the time step tnow
// (src/rk5.h:161-174), followed by the model's ExternalUpdate
// (src/aeif_cond_beta_multisynapse_kernel.h:190-226); returns true when the time step is
// complete.  `guard` counts the sub-steps of the current time step.
template <int MODEL, int PMAX, bool FIXED, int LM>
__device__ __forceinline__ bool aeif_substep(const AeifArgs &A, const SpikeOut &so, int i,
                                             const AeifQ<MODEL, PMAX, FIXED> &q, float *y, float &refr,
                                             double &x, float &h, long long tidx, double tnow,
                                             unsigned long long &nd, const float *smodel, int &guard) {
  const double x1 = tnow;
  const float hmax = (float)(x1 - x);
  nd += rk5_step<MODEL, PMAX, FIXED, LM>(x, y, h, A.hmin, A.hmin_acc, hmax, q, refr, so.status, smodel,
                                         A.learn);
  return aeif_external(A, so, i, q, y, refr, x, tidx, tnow, guard);
}

// After an accepted RK5 sub-step: whether the time step is complete, then the model's
// ExternalUpdate (src/aeif_cond_beta_multisynapse_kernel.h:190-226): state guards,
// refractoriness, spike and reset.
template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ bool aeif_external(const AeifArgs &A, const SpikeOut &so, int i,
                                              const AeifQ<MODEL, PMAX, FIXED> &q, float *y, float &refr,
                                              double x, long long tidx, double tnow, int &guard) {
  const double x1 = tnow;
  const bool end = (x >= x1 - (double)A.hmin);
  if (++guard > ck::max_substeps) {
    atomicOr(so.status, ST_RK5_TRIALS);
    return true;
  }
  if (y[0] < -1.0e3f) {
    y[0] = q.V_reset;
    y[1] = 0.0f;
    atomicOr(so.status, ST_NUMERIC);
    return end;
  }
  if (y[1] < -1.0e6f || y[1] > 1.0e6f) {
    y[0] = q.V_reset;
    y[1] = 0.0f;
    atomicOr(so.status, ST_NUMERIC);
    return end;
  }
  if (refr > 0.0f) {
    y[0] = q.V_reset;
    if (end) refr = __fsub_rn(refr, 1.0f);
  } else if (y[0] >= q.V_peak) {
    push_spike(so, A.srec, A.i0 + i, i, 1.0f, tidx, tnow);
    y[0] = q.V_reset;
    y[1] = __fadd_rn(y[1], q.b);
    refr = q.refr_steps;
  }
  return end;
}

// Records of the step (values after the update, before the fold).
// NVM: compile-time bound on nvar; the state is selected by comparisons so that it stays
// in registers.
template <int NVM>
__device__ __forceinline__ void write_records(const GroupRecord &R, const SpikeOut &so, int node, int i,
                                              const float *y, int nvar, float refr, long long row,
                                              long long tidx) {
  if (!R.first) return;
  const int c0 = R.first[i], c1 = R.first[i + 1];
  for (int c = c0; c < c1; c++) {
    const int2 rc = R.col[c];
    float v = 0.0f;
    if (rc.x < 0) v = (so.has_out_all[node] && so.last_tidx[node] == (int)tidx) ? so.last_height[node] : 0.0f;
    else if (rc.x == nvar) v = refr;
    else {
#pragma unroll
      for (int k = 0; k < NVM; k++)
        if (k == rc.x) v = y[k];
    }
    R.buf[(size_t)row * R.ncol + rc.y] = v;
  }
}

// End of step m: records, then the input fold (src/get_spike.cu:142-166) in FP64.
template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ void aeif_end_step(const AeifArgs &A, const SpikeOut &so, int i,
                                              const AeifQ<MODEL, PMAX, FIXED> &q, float *y, float refr,
                                              int m, const StepT &t, long long rec_it0, const double *apf,
                                              PoissonCache &pc) {
  typedef AeifShape<MODEL> S;
  const int np = q.ports();
  if (A.rec.first)
    write_records<2 + S::npv * PMAX>(A.rec, so, A.i0 + i, i, y, 2 + S::npv * np, refr, t.it - rec_it0, t.tidx);
  double in[PMAX];
  step_inputs_pf<PMAX>(in, apf, np, A.n, i, A.in, pc, m, t.tidx, t.tnow);
#pragma unroll
  for (int p = 0; p < PMAX; p++) {
    if (p < np && in[p] != 0.0) {
      const int iv = 2 + S::npv * p + S::in_var;
      y[iv] = (float)__fma_rn(in[p], (double)q.pw[p], (double)y[iv]);
    }
  }
}

template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ void aeif_load(const AeifArgs &A, int i, float *y, float &refr, double &x,
                                          float &h, int NV) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
#pragma unroll
  for (int v = 0; v < NVM; v++)
    if (v < NV) y[v] = A.var[(size_t)v * A.n + i];
  refr = A.refr[i];
  x = A.x[i];
  h = A.h[i];
}

template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ void aeif_store(const AeifArgs &A, int i, const float *y, float refr, double x,
                                           float h, int NV) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
#pragma unroll
  for (int v = 0; v < NVM; v++)
    if (v < NV) A.var[(size_t)v * A.n + i] = y[v];
  A.refr[i] = refr;
  A.x[i] = x;
  A.h[i] = h;
}

__device__ __forceinline__ void warp_add(unsigned long long *ctr, unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
}

// One iteration of the trial-per-iteration form: begin a step if none is open (k1 and the
// error scale), run one trial; after a rejection shrink h and return false (the step stays
// open); after an acceptance update x, h and y and run the ExternalUpdate.  Returns true
// when the time step is complete.  The operations of each step are those of rk5_step.
template <int MODEL, int PMAX, bool FIXED>
__device__ __forceinline__ bool aeif_tpi_iter(const AeifArgs &A, const SpikeOut &so, int i,
                                              const AeifQ<MODEL, PMAX, FIXED> &q, float *y, float &refr,
                                              double &x, float &h, const StepT &t, float *k1, float *iys,
                                              bool &open, int &trials, unsigned long long &nd, int &guard) {
  constexpr int NVM = 2 + AeifShape<MODEL>::npv * PMAX;
  const int NV = 2 + AeifShape<MODEL>::npv * q.ports();
  if (!open) {
    rk5_begin(y, h, q, refr, k1, iys);
    nd += 1;
    trials = 0;
    open = true;
  }
  float yn[NVM];
  const float err = rk5_trial(y, h, A.hmin, (float)(t.tnow - x), q, refr, k1, iys, yn);
  nd += 5;
  if (!(err <= 1.0f || h <= A.hmin_acc)) {
    if (++trials < ck::max_trials) {
      h = rk5_shrink(h, err);
      return false;
    }
    atomicOr(so.status, ST_RK5_TRIALS);
  }
  open = false;
  x += (double)h;
  h = rk5_grow(h, err, A.hmin);
#pragma unroll
  for (int v = 0; v < NVM; v++)
    if (v < NV) y[v] = yn[v];
  return aeif_external(A, so, i, q, y, refr, x, t.tidx, t.tnow, guard);
}

// Main aeif kernel: one thread per neuron, steps m = 0..M-1 of the batch.
// OCC = 1 caps the registers so that three 256-thread blocks fit on an SM (more warps
// in flight to hide the dependent FP32 latency, at the price of a few spills); OCC = 2
// (trial-per-iteration form, blocks of at most 128 threads) caps them at five 128-thread
// blocks per SM (96 registers: 20 warps, fewer spills).  Measured on the 1M network (RTF,
// 64-thread blocks): OCC = 0 (145 registers, 14 warps) 0.776, OCC = 1 (80, 24 warps, 204 B of
// spills) 0.683, OCC = 2 (96, 20 warps, 80 B) 0.649, and a 120-register cap without spills
// (16 warps) 0.661.
// TPI = true (plain controller only): one RK5 trial per loop iteration.  A lane whose
// trial is rejected retries in the next iteration, beside its neighbours' next trials,
// instead of holding its whole warp in a second trial (with ~4% of the trials rejected,
// most warps have a rejecting lane at most steps).  k1 and the error scale of the open
// step stay in registers across iterations; a lane is handed to the straggler kernel
// only between accepted steps, so every lane runs the same sequence of operations as
// in the step-at-once form and results are identical.
template <int MODEL, int PMAX, bool FIXED, int LM, int OCC = 0, bool UNI = false, bool TPI = false>
__global__ void __launch_bounds__(OCC == 2 ? 128 : 256, OCC == 1 ? 3 : (OCC == 2 ? 5 : 1))
    aeif_batch_kernel(const AeifArgs A, const SpikeOut so,
                                                         const Clock *clk, int k0, int M) {
  pdl_enter();
  typedef AeifShape<MODEL> S;
  constexpr int NVM = 2 + S::npv * PMAX;
  __shared__ float smodel[LM == LM_PROPOSE ? SM_NPAR : 1];
  if (LM == LM_PROPOSE) {
    for (int j = threadIdx.x; j < SM_NPAR; j += blockDim.x) smodel[j] = A.learn.model[j];
    __syncthreads();
  }
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nd = 0;
  if (i < A.hi) {
    AeifQ<MODEL, PMAX, FIXED> q;
    load_aeif_par<MODEL, PMAX, FIXED, UNI>(A, i, q);
    const int NV = 2 + S::npv * q.ports();
    float y[NVM];
    float refr, h;
    double x;
    aeif_load<MODEL, PMAX, FIXED>(A, i, y, refr, x, h, NV);
    const Clock cl = *clk;
    const long long rec_it0 = cl.rec_it0;
    int budget = A.budget > 0 ? A.budget : -1;
    PoissonCache pc;
    poisson_cache_load(A.in, i, pc);
    // One RK5 sub-step per iteration: a lane that needs extra sub-steps in one time step
    // does not hold the others of its warp in that step; they go on with their next step.
    int m = 0, guard = 0;
    bool deferred = false;
    StepT t = step_at(cl, k0, 0, A.dt);
    double apf[PMAX];
    acc_prefetch<PMAX>(apf, q.ports(), A.n, i, A.in, 0);
    if constexpr (TPI) {
      static_assert(LM == LM_PLAIN, "one trial per iteration is a form of the plain controller");
      float k1[NVM], iys[NVM];
      bool open = false;     // a step has begun (k1, iys valid) and no trial was accepted yet
      int trials = 0;
      while (m < M) {
        if (!open && budget == 0) {
          deferred = true;
          break;
        }
        if (budget > 0) budget--;
        if (aeif_tpi_iter(A, so, i, q, y, refr, x, h, t, k1, iys, open, trials, nd, guard)) {
          aeif_end_step(A, so, i, q, y, refr, m, t, rec_it0, apf, pc);
          guard = 0;
          if (++m < M) {
            t = step_at(cl, k0, m, A.dt);
            acc_prefetch<PMAX>(apf, q.ports(), A.n, i, A.in, m);
          }
        }
      }
    } else {
      while (m < M) {
        if (budget == 0) {
          deferred = true;
          break;
        }
        if (budget > 0) budget--;
        if (aeif_substep<MODEL, PMAX, FIXED, LM>(A, so, i, q, y, refr, x, h, t.tidx, t.tnow, nd, smodel,
                                                 guard)) {
          aeif_end_step(A, so, i, q, y, refr, m, t, rec_it0, apf, pc);
          guard = 0;
          if (++m < M) {
            t = step_at(cl, k0, m, A.dt);
            acc_prefetch<PMAX>(apf, q.ports(), A.n, i, A.in, m);
          }
        }
      }
    }
    aeif_store<MODEL, PMAX, FIXED>(A, i, y, refr, x, h, NV);
    if (deferred) {
      const int pos = atomicAdd(A.strag_cnt, 1);
      A.strag_list[pos] = make_int2(i, m);
    }
  }
  warp_add(A.nderiv, nd);
}

// Neurons the main kernel left unfinished (typically the few that spike in the batch)
// continue here from the step where they stopped, one per thread.  The kernel's length is
// the longest sub-step chain, so it gets all the registers it wants (151 for the benchmark's
// model; with 256-thread bounds it was held to 127: RTF 0.6490-0.6509 against 0.6456-0.6471).
// (The trial-per-iteration form measured 2.5% slower here than the step-at-once form: the
// lanes of this kernel are all in long sub-step chains.)
template <int MODEL, int PMAX, bool FIXED, int LM, bool UNI = false>
__global__ void __launch_bounds__(128, 1) aeif_straggler_kernel(const AeifArgs A, const SpikeOut so,
                                                             const Clock *clk, int k0, int M) {
  pdl_enter();
  typedef AeifShape<MODEL> S;
  constexpr int NVM = 2 + S::npv * PMAX;
  __shared__ float smodel[LM == LM_PROPOSE ? SM_NPAR : 1];
  if (LM == LM_PROPOSE) {
    for (int j = threadIdx.x; j < SM_NPAR; j += blockDim.x) smodel[j] = A.learn.model[j];
    __syncthreads();
  }
  const int cnt = *A.strag_cnt;
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  unsigned long long nd = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
    const int2 e = A.strag_list[j];
    const int i = e.x;
    AeifQ<MODEL, PMAX, FIXED> q;
    load_aeif_par<MODEL, PMAX, FIXED, UNI>(A, i, q);
    const int NV = 2 + S::npv * q.ports();
    float y[NVM];
    float refr, h;
    double x;
    aeif_load<MODEL, PMAX, FIXED>(A, i, y, refr, x, h, NV);
    PoissonCache pc;
    poisson_cache_load(A.in, i, pc);
    int m = e.y, guard = 0;
    StepT t = step_at(cl, k0, m, A.dt);
    double apf[PMAX];
    acc_prefetch<PMAX>(apf, q.ports(), A.n, i, A.in, m);
    while (m < M) {
      if (aeif_substep<MODEL, PMAX, FIXED, LM>(A, so, i, q, y, refr, x, h, t.tidx, t.tnow, nd, smodel, guard)) {
        aeif_end_step(A, so, i, q, y, refr, m, t, rec_it0, apf, pc);
        guard = 0;
        if (++m < M) {
          t = step_at(cl, k0, m, A.dt);
          acc_prefetch<PMAX>(apf, q.ports(), A.n, i, A.in, m);
        }
      }
    }
    aeif_store<MODEL, PMAX, FIXED>(A, i, y, refr, x, h, NV);
  }
  warp_add(A.nderiv, nd);
}

// Batch kernel, then the straggler kernel when a step budget is set; returns the
// number of kernels launched.
template <int MODEL, int PMAX, bool FIXED, int LM>
int launch_aeif_p(const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M, cudaStream_t st) {
  int tb = (A.threads == 64 || A.threads == 256) ? A.threads : 128;
  if (A.occupancy == 2 && tb > 128) tb = 128;   // the OCC = 2 variant is bounded to 128 threads
  dim3 grid((A.hi - A.lo + tb - 1) / tb), block(tb);
  bool done = false;
  if constexpr (LM == LM_PLAIN && FIXED) {
    if (A.trial_iter && A.occupancy == 2 && A.uniform) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 2, true, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.trial_iter && A.occupancy && A.uniform) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 1, true, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.trial_iter && A.uniform) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 0, true, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.trial_iter && A.occupancy) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 1, false, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.trial_iter) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 0, false, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.occupancy && A.uniform) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 1, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.occupancy) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 1>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    } else if (A.uniform) {
      launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 0, true>, grid, block, 0, st, A, so, clk, k0, M);
      done = true;
    }
  }
  if (!done) launch_k(aeif_batch_kernel<MODEL, PMAX, FIXED, LM, 0>, grid, block, 0, st, A, so, clk, k0, M);
  if (A.budget <= 0) return 1;
  const int nl = A.hi - A.lo;
  dim3 sgrid(nl < 128 * 148 * 4 ? (nl + 127) / 128 : 148 * 4), sblock(128);
  done = false;
  if constexpr (LM == LM_PLAIN && FIXED) {
    if (A.uniform) {
      launch_k(aeif_straggler_kernel<MODEL, PMAX, FIXED, LM, true>, sgrid, sblock, 0, st, A, so, clk, k0, M);
      done = true;
    }
  }
  if (!done) launch_k(aeif_straggler_kernel<MODEL, PMAX, FIXED, LM>, sgrid, sblock, 0, st, A, so, clk, k0, M);
  return 2;
}

}  // namespace ngpu
