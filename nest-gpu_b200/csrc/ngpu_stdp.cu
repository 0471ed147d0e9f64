// Spike-timing-dependent plasticity on the delivery CSR.
//
// Networks with plastic edges (synapse group > 0) advance one time step per batch, and
// each step T runs, around the step's delivery and update kernels:
//   before:  stamp reset at the 16-bit wrap points (src/nestgpu.cu:490-498,
//            src/rev_spike.cu:93-118);
//   after:   forward pass over the spikes arriving in T: each plastic edge records T as
//            its last arrival and is depressed against its target's last spike
//            (src/get_spike.cu:85-95); then the reverse pass: the plastic in-edges of
//            every node that spiked in T are potentiated against their last arrival
//            (src/rev_spike.cu:46-92).
// The delivery of T has already used the weights of the end of step T-1, as the
// reference's CollectSpike does before its update.  The weight rule is SynapseUpdate
// (src/syn_model.cu:43-56): STDPUpdate (src/stdp.cu:36-64) in FP64, or the linear test
// model (src/test_syn_model.cu:35-40).
#include <cuda_runtime.h>

#include "ngpu_aeif.cuh"
#include "ngpu_types.h"

namespace ngpu {

constexpr int MAX_SYN_DT = 16384;   // src/syn_model.h:33

__device__ __forceinline__ float synapse_update(int type, const float *par, float w, float Dt) {
  if (type == SYN_TEST) return __fadd_rn(w, __fmaf_rn(par[0], Dt, par[1]));
  const double tau_plus = par[0], tau_minus = par[1], lambda = par[2], alpha = par[3];
  const double mu_plus = par[4], mu_minus = par[5], Wmax = par[6];
  const double wd = w;
  double w1;
  if (Dt >= 0.0f) {
    const double fact = lambda * exp(-(double)Dt / tau_plus);
    w1 = wd + fact * Wmax * pow(1.0 - wd / Wmax, mu_plus);
  } else {
    const double fact = -alpha * lambda * exp((double)Dt / tau_minus);
    w1 = wd + fact * Wmax * pow(wd / Wmax, mu_minus);
  }
  w1 = w1 > 0.0 ? w1 : 0.0;
  w1 = w1 < Wmax ? w1 : Wmax;
  return (float)w1;
}

__device__ __forceinline__ long long step_tidx(const Clock *clk, int k0) {
  return clk->tidx_base + clk->it0 + k0 + 1;
}

// Up at T mod 2^16 = 0x8000: stamps of the older half become 0; down at 0: stamps of the
// other half become 0x8000.
__global__ void stdp_stamp_reset_kernel(const StdpArgs A, const Clock *clk, int k0) {
  const unsigned t16 = (unsigned)(step_tidx(clk, k0) & 0xffff);
  if (t16 != 0x8000u && t16 != 0u) return;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < A.n_pl;
       p += (long long)gridDim.x * blockDim.x) {
    const unsigned short s = A.stamp[p];
    if (t16 == 0x8000u && s >= 0x8000) A.stamp[p] = 0;
    if (t16 == 0u && s < 0x8000) A.stamp[p] = 0x8000;
  }
}

// One warp per delay group: its lanes take the spikes emitted T-1-(dmin+dd) steps ago.
__global__ void stdp_forward_kernel(const StdpArgs A, const Clock *clk, int k0) {
  const int dd = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (dd >= A.dspan) return;
  const long long T = step_tidx(clk, k0);
  const long long te = T - 1 - (A.dmin + dd);
  if (te < 1) return;
  const int rs = (int)(te % A.R);
  int cnt = A.ring_cnt[rs];
  cnt = cnt < A.cap ? cnt : A.cap;
  const unsigned short t16 = (unsigned short)(T & 0xffff);
  for (int j = threadIdx.x & 31; j < cnt; j += 32) {
    const int src = A.ring[(size_t)rs * A.cap + j].x;
    const size_t key = (size_t)src * A.dspan + dd;
    for (int p = A.pl_off[key]; p < A.pl_off[key + 1]; p++) {
      const PlasticEdge e = A.pl[p];
      A.stamp[p] = t16;
      const int last = A.last_tidx[e.target];
      if (last < 0) continue;   // the target has not spiked yet
      const long long Dt_int = T - last;
      if (Dt_int > 0 && Dt_int < MAX_SYN_DT) {
        const int g = e.group - 1;
        float &w = A.edge[e.pos].w;
        w = synapse_update(A.syn_type[g], A.syn_par + g * SYN_NPAR, w, -A.dt * (float)Dt_int);
      }
    }
  }
}

__global__ void stdp_reverse_kernel(const StdpArgs A, const Clock *clk, int k0) {
  const long long T = step_tidx(clk, k0);
  const unsigned short t16 = (unsigned short)(T & 0xffff);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.n_rev_nodes; r += gridDim.x * blockDim.x) {
    if ((long long)A.last_tidx[A.rev_node[r]] != T) continue;
    for (int q = A.rev_off[r]; q < A.rev_off[r + 1]; q++) {
      const int p = A.rev_id[q];
      const unsigned short Dt_int = (unsigned short)(t16 - A.stamp[p]);
      if (Dt_int < MAX_SYN_DT) {
        const PlasticEdge e = A.pl[p];
        const int g = e.group - 1;
        float &w = A.edge[e.pos].w;
        w = synapse_update(A.syn_type[g], A.syn_par + g * SYN_NPAR, w, A.dt * (float)Dt_int);
      }
    }
  }
}

// Spikes whose dendritic delay ends in step T reach their neuron's synapses: the reverse
// ring slot of T gives last_rev = T (set at the start of step T in the reference,
// src/spike_buffer.cu:314-316; only the plasticity passes after the update read it), and the
// slot is emptied for T + rev_R.
__global__ void rev_arrival_kernel(int *rev_ring, int *rev_cnt, int rev_R, int rev_cap, int *last_rev,
                                   const Clock *clk, int k0) {
  const long long T = step_tidx(clk, k0);
  const int rs = (int)(T % rev_R);
  int cnt = rev_cnt[rs];
  cnt = cnt < rev_cap ? cnt : rev_cap;
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) last_rev[rev_ring[(size_t)rs * rev_cap + j]] = (int)T;
  __syncthreads();
  if (threadIdx.x == 0) rev_cnt[rs] = 0;
}

int launch_rev_arrivals(int *rev_ring, int *rev_cnt, int rev_R, int rev_cap, int *last_rev, const Clock *clk,
                        int k0, cudaStream_t st) {
  rev_arrival_kernel<<<1, 256, 0, st>>>(rev_ring, rev_cnt, rev_R, rev_cap, last_rev, clk, k0);
  return 1;
}

int launch_stdp_reset(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st) {
  const long long nb = (A.n_pl + 255) / 256;
  stdp_stamp_reset_kernel<<<(int)(nb < 148 * 8 ? (nb > 0 ? nb : 1) : 148 * 8), 256, 0, st>>>(A, clk, k0);
  return 1;
}

int launch_stdp_forward(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st) {
  stdp_forward_kernel<<<(A.dspan + 3) / 4, 128, 0, st>>>(A, clk, k0);
  return 1;
}

int launch_stdp_reverse(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st) {
  const int nb = (A.n_rev_nodes + 127) / 128;
  stdp_reverse_kernel<<<nb < 148 * 8 ? (nb > 0 ? nb : 1) : 148 * 8, 128, 0, st>>>(A, clk, k0);
  return 1;
}

}  // namespace ngpu
