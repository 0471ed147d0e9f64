// CUDA kernels of the spiking engine (sm_100a).
//
// Time is advanced in batches of M steps, M <= the minimum synaptic delay in
// steps (a spike emitted in step s reaches its targets in step s+1+d, d >= dmin,
// so no spike emitted inside a batch affects the batch).  Per batch the graph runs:
//   1. deliver_batch_kernel: the spikes of the last dmax+1 steps walk their CSR
//      segments and add height*weight into the accumulator slot of the step in
//      which they arrive (FP64 atomics, one slot per step of the batch);
//   2. per node group one update kernel that integrates each neuron through all M
//      steps with its state in registers; at the end of every step it records,
//      then folds that step's arrivals and poiss_gen draws into the state, exactly
//      where the reference folds (src/nestgpu.cu:469-635: update, record,
//      CollectSpike, poiss_gen, GetSpikes); aeif neurons that need more RK5 steps
//      than a budget (those that spike) are finished by a straggler kernel, packed
//      densely, so their long step sequences do not stall whole warps.
#include <cub/block/block_scan.cuh>

#include <algorithm>

#include "ngpu_aeif.cuh"
#include "ngpu_math.cuh"
#include "ngpu_types.h"

namespace ngpu {

bool g_launch_pdl = false;
void set_launch_pdl(bool on) { g_launch_pdl = on; }

// ---------------------------------------------------------------------------
// iaf_psc_exp exact propagator (src/iaf_psc_exp.cu:85-110)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float iget(const IafArgs &A, int j, int i) {
  const float *p = A.parr[j];
  return p ? __ldg(p + i) : A.pval[j];
}

// Delivery at emission: the block adds the out-edges of node `src`, which spiked at time
// index `tidx`, into the accumulator ring.  The source's edges are contiguous in the CSR,
// delay group after delay group (group dd reaches the step with time index
// tidx + 1 + dmin + dd, as in the delivery kernel); thread t takes edges t, t + B, t + 2B, ...
// (B = block size, so each warp load is coalesced), four loads in flight before their
// reductions, and walks the delay groups (offsets staged in shared memory when they fit)
// as its edges advance.  FP64 reductions, so the sums equal those of the delivery kernel
// whatever the order.  Called by every thread of the block; returns the number of edges.
constexpr int PUSH_OFF_SMEM = 512;   // staged group offsets (dspan + 1 at most)

__device__ __noinline__ unsigned long long push_out_edges(const PushOut &po, int src, long long tidx, float height,
                                                          long long *s_off) {
  const long long base = (long long)src * po.dspan;
  const bool staged = po.dspan + 1 <= PUSH_OFF_SMEM;
  if (staged)
    for (int k = threadIdx.x; k <= po.dspan; k += blockDim.x) s_off[k] = __ldg(&po.ev_off[base + k]);
  __syncthreads();
  auto off = [&](int k) { return staged ? s_off[k] : __ldg(&po.ev_off[base + k]); };
  const long long s0 = off(0), s1 = off(po.dspan);
  const int B = blockDim.x;
  const uint2 *edge = reinterpret_cast<const uint2 *>(po.edge);
  int dd = 0;
  long long next = off(1);
  int slot = (int)((tidx + 1 + po.dmin) % po.R);
  for (long long e = s0 + threadIdx.x; e < s1; e += 4LL * B) {
    uint2 ew[4];
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (e + (long long)u * B < s1) ew[u] = __ldg(edge + e + (long long)u * B);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long eu = e + (long long)u * B;
      if (eu < s1) {
        while (eu >= next) {           // dd + 1 <= dspan: eu < s1 = off(dspan)
          dd++;
          next = off(dd + 1);
          if (++slot == po.R) slot = 0;
        }
        atomicAdd(&po.acc[(size_t)slot * po.stride + ew[u].x],
                  (double)__fmul_rn(height, __uint_as_float(ew[u].y)));
      }
    }
  }
  __syncthreads();                     // s_off is reused for the next spike
  return (unsigned long long)(s1 - s0);
}

__device__ __forceinline__ void iaf_neuron(const IafArgs &A, const SpikeOut &so, const Clock *clk, int k0,
                                           int M, int i) {
  const int n = A.n;
  float Iex = A.var[i], Iin = A.var[(size_t)n + i], V = A.var[2 * (size_t)n + i],
        refr = A.var[3 * (size_t)n + i];
  const float I_e = iget(A, IP_I_e, i), P20 = iget(A, IP_P20, i), P21ex = iget(A, IP_P21ex, i),
              P21in = iget(A, IP_P21in, i), P22 = iget(A, IP_P22, i), P11ex = iget(A, IP_P11ex, i),
              P11in = iget(A, IP_P11in, i), theta = iget(A, IP_Theta_rel, i),
              V_reset = iget(A, IP_V_reset_rel, i), refr_steps = iget(A, IP_refr_steps, i);
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  PoissonCache pc;
  poisson_cache_load(A.in, i, pc);
  for (int m = 0; m < M; m++) {
    const StepT t = step_at(cl, k0, m, A.dt);
    double apf[2];
    acc_prefetch<2>(apf, 2, n, i, A.in, m);
    if (refr > 0.0f) {
      refr = __fsub_rn(refr, 1.0f);
    } else {
      V = __fmaf_rn(I_e, P20, __fmaf_rn(Iin, P21in, __fmaf_rn(Iex, P21ex, __fmul_rn(V, P22))));
    }
    Iex = __fmul_rn(Iex, P11ex);
    Iin = __fmul_rn(Iin, P11in);
    if (V >= theta) {
      push_spike(so, A.srec, A.i0 + i, i, 1.0f, t.tidx, t.tnow);
      V = V_reset;
      refr = refr_steps;
    }
    if (A.rec.first) {
      const float yr[4] = {Iex, Iin, V, refr};
      write_records<4>(A.rec, so, A.i0 + i, i, yr, 4, refr, t.it - rec_it0, t.tidx);
    }
    double in[2];
    step_inputs_pf<2>(in, apf, 2, n, i, A.in, pc, m, t.tidx, t.tnow);
    if (in[0] != 0.0) Iex = (float)__fma_rn(in[0], 1.0, (double)Iex);
    if (in[1] != 0.0) Iin = (float)__fma_rn(in[1], 1.0, (double)Iin);
  }
  A.var[i] = Iex;
  A.var[(size_t)n + i] = Iin;
  A.var[2 * (size_t)n + i] = V;
  A.var[3 * (size_t)n + i] = refr;
}

// iaf_neuron with delivery at emission: every thread of the block runs the loop (`valid` false
// past the group's end) so that after each step the block delivers the out-edges of its
// neurons that spiked; the input slot of a step is the ring slot of its time index.  The
// arithmetic of the step is iaf_neuron's.
__device__ __forceinline__ void iaf_neuron_push(const IafArgs &A, const SpikeOut &so, const PushOut &po,
                                                const Clock *clk, int k0, int M, int i, bool valid, int *s_src,
                                                int *s_n, long long *s_off) {
  const int n = A.n;
  float Iex = 0.0f, Iin = 0.0f, V = 0.0f, refr = 0.0f, I_e = 0.0f, P20 = 0.0f, P21ex = 0.0f, P21in = 0.0f,
        P22 = 0.0f, P11ex = 0.0f, P11in = 0.0f, theta = 0.0f, V_reset = 0.0f, refr_steps = 0.0f;
  PoissonCache pc;
  pc.e0 = pc.e1 = 0;
  if (valid) {
    Iex = A.var[i];
    Iin = A.var[(size_t)n + i];
    V = A.var[2 * (size_t)n + i];
    refr = A.var[3 * (size_t)n + i];
    I_e = iget(A, IP_I_e, i);
    P20 = iget(A, IP_P20, i);
    P21ex = iget(A, IP_P21ex, i);
    P21in = iget(A, IP_P21in, i);
    P22 = iget(A, IP_P22, i);
    P11ex = iget(A, IP_P11ex, i);
    P11in = iget(A, IP_P11in, i);
    theta = iget(A, IP_Theta_rel, i);
    V_reset = iget(A, IP_V_reset_rel, i);
    refr_steps = iget(A, IP_refr_steps, i);
    poisson_cache_load(A.in, i, pc);
  }
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  unsigned long long nev = 0;
  for (int m = 0; m < M; m++) {
    const StepT t = step_at(cl, k0, m, A.dt);
    const int slot = (int)(t.tidx % po.R);
    double apf[2] = {0.0, 0.0};
    if (valid) acc_prefetch<2>(apf, 2, n, i, A.in, slot);
    if (refr > 0.0f) {
      refr = __fsub_rn(refr, 1.0f);
    } else {
      V = __fmaf_rn(I_e, P20, __fmaf_rn(Iin, P21in, __fmaf_rn(Iex, P21ex, __fmul_rn(V, P22))));
    }
    Iex = __fmul_rn(Iex, P11ex);
    Iin = __fmul_rn(Iin, P11in);
    const bool spike = valid && V >= theta;
    if (spike) {
      push_spike<false>(so, A.srec, A.i0 + i, i, 1.0f, t.tidx, t.tnow);
      V = V_reset;
      refr = refr_steps;
    }
    // the block's spikes of this step, then their out-edges, one spike after the other
    if (threadIdx.x == 0) *s_n = 0;
    __syncthreads();
    if (spike) s_src[atomicAdd(s_n, 1)] = A.i0 + i;
    __syncthreads();
    const int ns = *s_n;
    for (int j = 0; j < ns; j++) nev += push_out_edges(po, s_src[j], t.tidx, 1.0f, s_off);
    __syncthreads();
    if (valid && A.rec.first) {
      const float yr[4] = {Iex, Iin, V, refr};
      write_records<4>(A.rec, so, A.i0 + i, i, yr, 4, refr, t.it - rec_it0, t.tidx);
    }
    if (valid) {
      double in[2];
      step_inputs_pf<2>(in, apf, 2, n, i, A.in, pc, slot, t.tidx, t.tnow);
      if (in[0] != 0.0) Iex = (float)__fma_rn(in[0], 1.0, (double)Iex);
      if (in[1] != 0.0) Iin = (float)__fma_rn(in[1], 1.0, (double)Iin);
    }
  }
  if (valid) {
    A.var[i] = Iex;
    A.var[(size_t)n + i] = Iin;
    A.var[2 * (size_t)n + i] = V;
    A.var[3 * (size_t)n + i] = refr;
  }
  if (threadIdx.x == 0 && nev) atomicAdd(po.n_events, nev);
}

__global__ void __launch_bounds__(256, 3) iaf_batch_kernel(const IafArgs A, const SpikeOut so,
                                                        const Clock *clk, int k0, int M) {
  pdl_enter();
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < A.hi) iaf_neuron(A, so, clk, k0, M, i);
}

// Delivery at emission: every thread of the block runs the step loop.
__global__ void __launch_bounds__(256, 3) iaf_push_batch_kernel(const IafArgs A, const SpikeOut so, const PushOut po,
                                                             const Clock *clk, int k0, int M) {
  pdl_enter();
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ int s_src[256];
  __shared__ int s_n;
  __shared__ long long s_off[PUSH_OFF_SMEM];
  iaf_neuron_push(A, so, po, clk, k0, M, i, i < A.hi, s_src, &s_n, s_off);
}

// All iaf_psc_exp groups in one launch (a network of several populations would
// otherwise pay one launch per population and step): block b serves group g with
// blk0[g] <= b < blk0[g+1]; the groups' argument blocks are in device memory.
// Three 256-thread blocks per SM (80 registers): 113k neurons fit in one wave, which
// keeps the 77k-neuron microcircuit's 302 blocks from spilling into a second wave.
__global__ void __launch_bounds__(256, 3) iaf_multi_kernel(const IafArgs *tab, const int *blk0, int ngroups,
                                                        const SpikeOut so, const Clock *clk, int k0, int M) {
  pdl_enter();
  int lo = 0, hi = ngroups;   // largest g with blk0[g] <= blockIdx.x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (blk0[mid] <= (int)blockIdx.x) lo = mid; else hi = mid;
  }
  const IafArgs &A = tab[lo];
  const int i = A.lo + ((int)blockIdx.x - blk0[lo]) * blockDim.x + threadIdx.x;
  if (i < A.hi) iaf_neuron(A, so, clk, k0, M, i);
}

// The multi-group launch with delivery at emission.
__global__ void __launch_bounds__(256, 3) iaf_push_multi_kernel(const IafArgs *tab, const int *blk0, int ngroups,
                                                             const SpikeOut so, const PushOut po, const Clock *clk,
                                                             int k0, int M) {
  pdl_enter();
  int lo = 0, hi = ngroups;   // largest g with blk0[g] <= blockIdx.x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (blk0[mid] <= (int)blockIdx.x) lo = mid; else hi = mid;
  }
  const IafArgs &A = tab[lo];
  const int i = A.lo + ((int)blockIdx.x - blk0[lo]) * blockDim.x + threadIdx.x;
  __shared__ int s_src[256];
  __shared__ int s_n;
  __shared__ long long s_off[PUSH_OFF_SMEM];
  iaf_neuron_push(A, so, po, clk, k0, M, i, i < A.hi, s_src, &s_n, s_off);
}

// ---------------------------------------------------------------------------
// parrot_neuron (src/parrot_neuron.cu:60-82): the input of a step (port 0, weight 1) is
// repeated as a spike in the next one (height 1, or the input with hold_spike_height);
// port 1 has weight 0 (its spikes only reach plastic synapses).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) parrot_batch_kernel(const ParrotArgs A, const SpikeOut so, const Clock *clk,
                                                           int k0, int M) {
  pdl_enter();
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.hi) return;
  const int n = A.n;
  float in0 = A.var[i], dummy = A.var[(size_t)n + i], V = A.var[2 * (size_t)n + i];
  const bool hold = A.hold[i] != 0.0f;
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  PoissonCache pc;
  poisson_cache_load(A.in, i, pc);
  for (int m = 0; m < M; m++) {
    const StepT t = step_at(cl, k0, m, A.dt);
    double apf[2];
    acc_prefetch<2>(apf, 2, n, i, A.in, m);
    const float sh = in0;
    V = sh;
    if (sh != 0.0f) {
      in0 = 0.0f;
      push_spike(so, A.srec, A.i0 + i, i, hold ? sh : 1.0f, t.tidx, t.tnow);
    }
    if (A.rec.first) {
      const float yr[3] = {in0, dummy, V};
      write_records<3>(A.rec, so, A.i0 + i, i, yr, 3, 0.0f, t.it - rec_it0, t.tidx);
    }
    double in[2];
    step_inputs_pf<2>(in, apf, 2, n, i, A.in, pc, m, t.tidx, t.tnow);
    if (in[0] != 0.0) in0 = (float)__fma_rn(in[0], 1.0, (double)in0);
  }
  A.var[i] = in0;
  A.var[(size_t)n + i] = dummy;
  A.var[2 * (size_t)n + i] = V;
}

// ---------------------------------------------------------------------------
// spike_detector (src/spike_detector.cu:28-50): the input of a step (one port, weight 1)
// becomes spike_height in the next one (1, or the input itself with hold_spike_height);
// it emits nothing.  State [2][n]: input_spike_height, spike_height.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) spike_det_batch_kernel(const ParrotArgs A, const SpikeOut so,
                                                              const Clock *clk, int k0, int M) {
  pdl_enter();
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.hi) return;
  const int n = A.n;
  float in0 = A.var[i], sh = A.var[(size_t)n + i];
  const bool hold = A.hold[i] != 0.0f;
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  PoissonCache pc;
  poisson_cache_load(A.in, i, pc);
  for (int m = 0; m < M; m++) {
    const StepT t = step_at(cl, k0, m, A.dt);
    double apf[1];
    acc_prefetch<1>(apf, 1, n, i, A.in, m);
    sh = in0;
    if (sh != 0.0f) {
      if (!hold) sh = 1.0f;
      in0 = 0.0f;
    }
    if (A.rec.first) {
      const float yr[2] = {in0, sh};
      write_records<2>(A.rec, so, A.i0 + i, i, yr, 2, 0.0f, t.it - rec_it0, t.tidx);
    }
    double in[1];
    step_inputs_pf<1>(in, apf, 1, n, i, A.in, pc, m, t.tidx, t.tnow);
    if (in[0] != 0.0) in0 = (float)__fma_rn(in[0], 1.0, (double)in0);
  }
  A.var[i] = in0;
  A.var[(size_t)n + i] = sh;
}

// ---------------------------------------------------------------------------
// spike_generator (src/spike_generator.cu:49-67): compares against the per-call
// step counter, at most one spike per step.
// ---------------------------------------------------------------------------
__global__ void spike_gen_batch_kernel(const SpikeGenArgs A, const SpikeOut so, const Clock *clk, int k0,
                                       int M) {
  pdl_enter();
  const int i = A.lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.hi) return;
  const int e0 = A.off[i], e1 = A.off[i + 1];
  int nx = A.next[i];
  const Clock cl = *clk;
  const long long rec_it0 = cl.rec_it0;
  for (int m = 0; m < M; m++) {
    const StepT t = step_at(cl, k0, m, A.dt);
    const int e = e0 + nx;
    if (e < e1 && (long long)A.tidx[e] == t.it) {
      push_spike(so, A.srec, A.i0 + i, i, A.height[e], t.tidx, t.tnow);
      nx++;
    }
    if (A.rec.first) write_records<0>(A.rec, so, A.i0 + i, i, nullptr, 0, 0.0f, t.it - rec_it0, t.tidx);
  }
  A.next[i] = nx;
}

// ---------------------------------------------------------------------------
// Delivery of the spikes arriving during a batch.  Work items are (emission step,
// spike, delay group) with arrival step in the batch; a group of G lanes (G = 8, 16
// or 32: short segments waste fewer lanes with small G) per item streams the item's
// CSR segment with coalesced 8-byte loads and FP64 atomics into the accumulator
// slot of the arrival step.  Items are numbered arrival-step-major, so the items in
// flight at any moment reduce into one or two slots and those stay in L2 even when
// all slots of a batch together do not.
// ---------------------------------------------------------------------------
constexpr int DELIVER_THREADS = 256;
constexpr int MAX_PAIRS = 8192;     // dspan * M

typedef cub::BlockScan<int, DELIVER_THREADS> DeliverScan;

// The delivery of one batch by block `block` of `nblocks`; s_pref holds dspan*M+1 ints.
template <int G, bool AGG = false, bool PF = false>
__device__ __forceinline__ void deliver_batch(const DeliverArgs &A, const Clock *clk, int k0, int M, int *s_pref,
                                              typename DeliverScan::TempStorage &scan_tmp, int block,
                                              int nblocks) {
  typedef DeliverScan Scan;
  const long long t_first = clk->tidx_base + clk->it0 + k0 + 1;   // time index of step 0
  const int npairs = A.dspan * M;
  const int per = (npairs + DELIVER_THREADS - 1) / DELIVER_THREADS;
  int local = 0;
  const int b0 = threadIdx.x * per;
  for (int j = 0; j < per; j++) {
    const int pr = b0 + j;
    if (pr < npairs) {
      const int m = pr / A.dspan, dd = pr - m * A.dspan;
      const long long te = t_first + m - 1 - (A.dmin + dd);   // emission step
      int c = 0;
      if (te >= 1) {
        c = A.ring_cnt[(int)(te % A.R)];
        c = c < A.cap ? c : A.cap;
      }
      s_pref[pr + 1] = c;
      local += c;
    }
  }
  int excl;
  Scan(scan_tmp).ExclusiveSum(local, excl);
  __syncthreads();
  for (int j = 0; j < per; j++) {
    const int pr = b0 + j;
    if (pr < npairs) {
      excl += s_pref[pr + 1];
      s_pref[pr + 1] = excl;
    }
  }
  if (threadIdx.x == 0) s_pref[0] = 0;
  __syncthreads();
  const int total = s_pref[npairs];
  if (block == 0) {
    // ring slots of this batch's steps start empty (their previous steps are older than
    // any emission step read here because R >= M + dmax + 3); straggler lists start empty
    for (int m = threadIdx.x; m < M; m += blockDim.x) A.ring_cnt[(int)((t_first + m) % A.R)] = 0;
    for (int g = threadIdx.x; g < A.n_strag; g += blockDim.x) A.strag_cnt[g] = 0;
    if (A.xch && threadIdx.x == 0) A.xch[0].x = 0;
  }
  const int sub = threadIdx.x & (G - 1);
  const int grp = (block * DELIVER_THREADS + threadIdx.x) / G;
  const int ngrp = (nblocks * DELIVER_THREADS) / G;
  unsigned long long nev = 0;
  // Work item `item`: its (arrival step, delay) pair, the spike's height and the segment.
  struct Item {
    int m;
    float height;
    long long e0, e1;
  };
  auto fetch = [&](int item) {
    int lo = 0, hi = npairs;   // pair with s_pref[pr] <= item < s_pref[pr+1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_pref[mid] <= item) lo = mid; else hi = mid;
    }
    const int m = lo / A.dspan, dd = lo - m * A.dspan;
    const int j = item - s_pref[lo];
    const long long te = t_first + m - 1 - (A.dmin + dd);
    // segment offsets and edges are written by no kernel that delivers (the persistent loop
    // writes ring entries between its deliveries): read-only path for those two
    const int2 sp = A.ring[(size_t)(te % A.R) * A.cap + j];
    const size_t key = (size_t)sp.x * A.dspan + dd;
    Item it;
    it.m = m;
    it.height = __int_as_float(sp.y);
    it.e0 = __ldg(&A.ev_off[key]);
    it.e1 = __ldg(&A.ev_off[key + 1]);
    return it;
  };
  auto deliver = [&](const Item &it) {
    const long long e0 = it.e0, e1 = it.e1;
    const float height = it.height;
    double *acc = A.acc + (size_t)it.m * A.slot_stride;
    if constexpr (AGG) {
      // warp-aggregated reductions (G = 32: the warp is one work group, so this loop is
      // warp-uniform): lanes whose edges share a target add their products first and the
      // lowest of them issues one reduction.  FP64 sums of these products are exact, so the
      // result does not depend on how they are grouped.
      static_assert(G == 32, "warp aggregation needs one segment per warp");
      const int lane = threadIdx.x & 31;
      for (long long base = e0; base < e1; base += 32) {
        const long long e = base + lane;
        const bool valid = e < e1;
        uint2 ew = make_uint2(0xffffffffu, 0u);
        if (valid) ew = __ldg(reinterpret_cast<const uint2 *>(A.edge + e));
        double v = valid ? (double)__fmul_rn(height, __uint_as_float(ew.y)) : 0.0;
        const unsigned peers = __match_any_sync(0xffffffffu, ew.x);
        if (__any_sync(0xffffffffu, __popc(peers) > 1)) {
          double sum = 0.0;
          for (int k = 0; k < 32; k++) {
            const double o = __shfl_sync(0xffffffffu, v, k);
            if ((peers >> k) & 1u) sum += o;
          }
          v = sum;
        }
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&acc[ew.x], v);
      }
    } else {
      for (long long e = e0 + sub; e < e1; e += G) {
        const uint2 ew = __ldg(reinterpret_cast<const uint2 *>(A.edge + e));
        atomicAdd(&acc[ew.x], (double)__fmul_rn(height, __uint_as_float(ew.y)));
      }
    }
    if (sub == 0) nev += (unsigned long long)(e1 - e0);
  };
  if constexpr (PF) {
    // software pipeline: the next item's ring entry and segment offsets are loaded before
    // this item's edges, so their dependent latencies overlap this item's traffic
    int item = grp;
    Item cur;
    if (item < total) cur = fetch(item);
    while (item < total) {
      const int next = item + ngrp;
      Item nxt;
      if (next < total) nxt = fetch(next);
      deliver(cur);
      cur = nxt;
      item = next;
    }
  } else {
    for (int item = grp; item < total; item += ngrp) deliver(fetch(item));
  }
  // one counter update per block
  for (int o = 16; o > 0; o >>= 1) nev += __shfl_down_sync(0xffffffffu, nev, o);
  __shared__ unsigned long long s_nev;
  if (threadIdx.x == 0) s_nev = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0 && nev) atomicAdd(&s_nev, nev);
  __syncthreads();
  if (threadIdx.x == 0 && s_nev) atomicAdd(A.n_events, s_nev);
  __syncthreads();
}

template <int G, bool AGG = false, bool PF = false>
__global__ void __launch_bounds__(DELIVER_THREADS) deliver_batch_kernel(const DeliverArgs A,
                                                                        const Clock *clk, int k0, int M) {
  pdl_enter();
  extern __shared__ int s_pref[];   // npairs + 1 prefix sums over (delay group, arrival step)
  __shared__ typename DeliverScan::TempStorage scan_tmp;
  deliver_batch<G, AGG, PF>(A, clk, k0, M, s_pref, scan_tmp, blockIdx.x, gridDim.x);
}

__global__ void clock_advance_kernel(Clock *clk, int K) {
  pdl_enter();
  clk->it0 += K;
}

// ---------------------------------------------------------------------------
// Persistent step loop for networks whose neurons are all iaf_psc_exp.  One
// cooperative launch (all blocks co-resident) advances K steps in batches of M:
// delivery, grid barrier, update of every population, grid barrier.  With a minimum
// delay of one step (M = 1) this replaces two launches per step.
// ---------------------------------------------------------------------------
// Counting barrier over the blocks of the launch.  Waits are bounded: after 2^24 polls
// a block records a timeout in the status word, and every later barrier of the launch
// returns false at once, so the kernel ends instead of waiting for ever.
__device__ __forceinline__ bool grid_barrier(GridBarrier *bar, unsigned nblocks, unsigned *status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = (((volatile unsigned *)status)[0] & ST_BARRIER_TIMEOUT) ? 0 : 1;
    if (ok) {
      const unsigned g = ((volatile unsigned *)&bar->gen)[0];
      __threadfence();
      if (atomicAdd(&bar->count, 1u) + 1u == nblocks) {
        atomicExch(&bar->count, 0u);
        __threadfence();
        atomicAdd(&bar->gen, 1u);
      } else {
        long long polls = 0;
        while (((volatile unsigned *)&bar->gen)[0] == g) {
          if (++polls > (1LL << 24)) {
            atomicOr(status, ST_BARRIER_TIMEOUT);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int G>
__global__ void __launch_bounds__(DELIVER_THREADS) persistent_iaf_kernel(
    const DeliverArgs D, const IafArgs *tab, const int *first, int ngroups, const SpikeOut so, const Clock *clk,
    int K, int M, GridBarrier *bar, int extra) {
  extern __shared__ int s_pref[];
  __shared__ typename DeliverScan::TempStorage scan_tmp;
  const int total_n = first[ngroups];
  const unsigned nb = gridDim.x + (unsigned)extra;   // extra > 0 only in the timeout test
  for (int k0 = 0; k0 < K; k0 += M) {
    const int mb = (K - k0 < M) ? K - k0 : M;
    deliver_batch<G>(D, clk, k0, mb, s_pref, scan_tmp, blockIdx.x, gridDim.x);
    if (!grid_barrier(bar, nb, so.status)) return;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total_n; gi += gridDim.x * blockDim.x) {
      int lo = 0, hi = ngroups;   // group with first[g] <= gi < first[g+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= gi) lo = mid; else hi = mid;
      }
      iaf_neuron(tab[lo], so, clk, k0, mb, gi - first[lo]);
    }
    if (!grid_barrier(bar, nb, so.status)) return;
  }
}

// Cooperative launch of the persistent loop over `steps` steps; the grid is the number of
// blocks that fit on the GPU at once (at most `max_blocks`).
int launch_persistent_iaf(const DeliverArgs &D, int group, const IafArgs *tab, const int *first, int ngroups,
                          const SpikeOut &so, const Clock *clk, int steps, int M, GridBarrier *bar, int max_blocks,
                          int barrier_extra, cudaStream_t st) {
  const size_t smem = (size_t)(D.dspan * M + 1) * sizeof(int);
  void *fn = group == 8 ? (void *)persistent_iaf_kernel<8>
                        : group == 16 ? (void *)persistent_iaf_kernel<16> : (void *)persistent_iaf_kernel<32>;
  int dev = 0, n_sm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, DELIVER_THREADS, smem);
  int nblocks = n_sm * per_sm;
  if (max_blocks > 0 && nblocks > max_blocks) nblocks = max_blocks;
  if (nblocks < 1) return -1;
  DeliverArgs d = D;
  const IafArgs *t = tab;
  const int *f = first;
  int ng = ngroups;
  SpikeOut s = so;
  const Clock *c = clk;
  int k = steps, m = M;
  GridBarrier *b = bar;
  int x = barrier_extra;
  void *args[] = {&d, &t, &f, &ng, &s, &c, &k, &m, &b, &x};
  if (cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(DELIVER_THREADS), args, smem, st) != cudaSuccess)
    return -1;
  return 1;
}

// ---------------------------------------------------------------------------
// Host-side launchers.  Each returns the number of kernels it launched.
// ---------------------------------------------------------------------------
template <int MODEL>
static int launch_aeif_m(const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                         cudaStream_t st) {
  switch (A.nport) {
  case 1: return launch_aeif_p<MODEL, 1, true, LM_PLAIN>(A, so, clk, k0, M, st);
  case 2: return launch_aeif_p<MODEL, 2, true, LM_PLAIN>(A, so, clk, k0, M, st);
  case 3: return launch_aeif_p<MODEL, 3, true, LM_PLAIN>(A, so, clk, k0, M, st);
  case 4: return launch_aeif_p<MODEL, 4, true, LM_PLAIN>(A, so, clk, k0, M, st);
  default: return launch_aeif_p<MODEL, MAX_PORT, false, LM_PLAIN>(A, so, clk, k0, M, st);
  }
}

int launch_aeif_learn(int model, const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                      cudaStream_t st);

int launch_aeif(int model, const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                cudaStream_t st) {
  if (A.hi <= A.lo) return 0;
  if (A.learn.mode != LM_PLAIN) return launch_aeif_learn(model, A, so, clk, k0, M, st);
  switch (model) {
  case M_AEIF_COND_BETA: return launch_aeif_m<M_AEIF_COND_BETA>(A, so, clk, k0, M, st);
  case M_AEIF_COND_ALPHA: return launch_aeif_m<M_AEIF_COND_ALPHA>(A, so, clk, k0, M, st);
  case M_AEIF_PSC_EXP: return launch_aeif_m<M_AEIF_PSC_EXP>(A, so, clk, k0, M, st);
  case M_AEIF_PSC_ALPHA: return launch_aeif_m<M_AEIF_PSC_ALPHA>(A, so, clk, k0, M, st);
  }
  return 0;
}

int launch_iaf(const IafArgs &A, const SpikeOut &so, const PushOut *po, const Clock *clk, int k0, int M,
               cudaStream_t st) {
  if (A.hi <= A.lo) return 0;
  const dim3 g((A.hi - A.lo + 255) / 256), b(256);
  if (po) launch_k(iaf_push_batch_kernel, g, b, 0, st, A, so, *po, clk, k0, M);
  else launch_k(iaf_batch_kernel, g, b, 0, st, A, so, clk, k0, M);
  return 1;
}

int launch_iaf_multi(const IafArgs *tab, const int *blk0, int ngroups, int nblocks, const SpikeOut &so,
                     const PushOut *po, const Clock *clk, int k0, int M, cudaStream_t st) {
  if (nblocks <= 0) return 0;
  if (po) launch_k(iaf_push_multi_kernel, dim3(nblocks), dim3(256), 0, st, tab, blk0, ngroups, so, *po, clk, k0, M);
  else launch_k(iaf_multi_kernel, dim3(nblocks), dim3(256), 0, st, tab, blk0, ngroups, so, clk, k0, M);
  return 1;
}

int launch_spike_det(const ParrotArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M, cudaStream_t st) {
  if (A.hi <= A.lo) return 0;
  launch_k(spike_det_batch_kernel, dim3((A.hi - A.lo + 255) / 256), dim3(256), 0, st, A, so, clk, k0, M);
  return 1;
}

int launch_parrot(const ParrotArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M, cudaStream_t st) {
  if (A.hi <= A.lo) return 0;
  launch_k(parrot_batch_kernel, dim3((A.hi - A.lo + 255) / 256), dim3(256), 0, st, A, so, clk, k0, M);
  return 1;
}

int launch_spike_gen(const SpikeGenArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                     cudaStream_t st) {
  if (A.hi <= A.lo) return 0;
  launch_k(spike_gen_batch_kernel, dim3((A.hi - A.lo + 255) / 256), dim3(256), 0, st, A, so, clk, k0, M);
  return 1;
}

int launch_deliver(const DeliverArgs &A, int n_blocks, int group, const Clock *clk, int k0, int M,
                   cudaStream_t st) {
  const size_t smem = (size_t)(A.dspan * M + 1) * sizeof(int);
  const dim3 g(n_blocks), b(DELIVER_THREADS);
  if (A.prefetch) {
    if (group == 8) launch_k(deliver_batch_kernel<8, false, true>, g, b, smem, st, A, clk, k0, M);
    else if (group == 16) launch_k(deliver_batch_kernel<16, false, true>, g, b, smem, st, A, clk, k0, M);
    else if (A.aggregate) launch_k(deliver_batch_kernel<32, true, true>, g, b, smem, st, A, clk, k0, M);
    else launch_k(deliver_batch_kernel<32, false, true>, g, b, smem, st, A, clk, k0, M);
  } else {
    if (group == 8) launch_k(deliver_batch_kernel<8>, g, b, smem, st, A, clk, k0, M);
    else if (group == 16) launch_k(deliver_batch_kernel<16>, g, b, smem, st, A, clk, k0, M);
    else if (A.aggregate) launch_k(deliver_batch_kernel<32, true>, g, b, smem, st, A, clk, k0, M);
    else launch_k(deliver_batch_kernel<32>, g, b, smem, st, A, clk, k0, M);
  }
  return 1;
}

// Partitioned network: the spikes the other processes' neurons emitted in the batch
// (recv[q] = their exchange buffers, q = 0 .. world-1, this process's own block skipped) go
// into this process's ring when their source has out-edges to neurons simulated here.
__global__ void exchange_unpack_kernel(SpikeOut so, const int4 *recv, int xch_cap, int world, int rank) {
  const int q = blockIdx.x;
  if (q == rank || q >= world) return;
  const int4 *b = recv + (size_t)q * (xch_cap + 1);
  const int n = min(b[0].x, xch_cap);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const int4 e = b[1 + j];
    if (!so.has_out[e.x]) continue;
    const int slot = (int)((long long)e.z % so.R);
    const int pos = atomicAdd(&so.ring_cnt[slot], 1);
    if (pos < so.cap) so.ring[(size_t)slot * so.cap + pos] = make_int2(e.x, e.y);
    else atomicOr(so.status, ST_RING_OVERFLOW);
  }
}

int launch_exchange_unpack(const SpikeOut &so, const int4 *recv, int xch_cap, int world, int rank,
                           cudaStream_t st) {
  exchange_unpack_kernel<<<world, 256, 0, st>>>(so, recv, xch_cap, world, rank);
  return 1;
}

int launch_clock_advance(Clock *clk, int K, cudaStream_t st) {
  launch_k(clock_advance_kernel, dim3(1), dim3(1), 0, st, clk, K);
  return 1;
}

int deliver_max_pairs() { return MAX_PAIRS; }

}  // namespace ngpu
