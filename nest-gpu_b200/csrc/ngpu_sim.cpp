// Calibration into the device layout and the CUDA-graph step loop.
//
// Device layout (structure of arrays, one allocation per array):
//   per group   state [nvar][n] float, aeif x [n] double, h [n] float, refractory [n] float;
//               derived parameters: uniform -> kernel argument, else [n] float array;
//               target-major poiss_gen in-edges (pin_off [n+1], PoissonIn [..]).
//   global      acc [sum(n*nport)] double (spike input of the previous step);
//               recurrent edges sorted by (source, delay): EdgeW {acc index, weight},
//               ev_off [n_nodes*dspan + 1] int64 segment starts;
//               spike ring [R][cap] (node, height) with counts [R], R = max delay + 3;
//               per node has_out, last spike time index and height; clock; counters.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "ngpu_engine.h"

namespace ngpu {

enum { A_V_th = 0, A_Delta_T, A_g_L, A_E_L, A_C_m, A_a, A_b, A_tau_w, A_I_e, A_V_peak,
       A_V_reset, A_t_ref, A_refractory_step, A_den_delay, A_NSCAL };
enum { I_tau_m = 0, I_C_m, I_E_L, I_I_e, I_Theta_rel, I_V_reset_rel, I_tau_ex, I_tau_in, I_t_ref,
       I_den_delay, I_P20, I_P11ex, I_P11in, I_P21ex, I_P21in, I_P22, I_NPAR };
enum { PG_rate = 0, PG_origin, PG_start, PG_stop };

static bool is_aeif(int m) { return m <= M_AEIF_PSC_ALPHA; }
static int n_port_par(int m) {
  switch (m) {
  case M_AEIF_COND_BETA: return 4;
  case M_AEIF_COND_ALPHA: return 3;
  case M_AEIF_PSC_EXP: return 1;
  case M_AEIF_PSC_ALPHA: return 2;
  default: return 0;
  }
}
static int n_port_var(int m) { return m == M_AEIF_PSC_EXP ? 1 : 2; }

static void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw NgpuError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

template <class T> T *Engine::dalloc(size_t n) {
  T *p = nullptr;
  if (n == 0) n = 1;
  cuda_check(cudaMalloc((void **)&p, n * sizeof(T)), "cudaMalloc");
  allocs_.push_back(p);
  return p;
}

void Engine::free_device() {
  for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
  for (void *p : allocs_) cudaFree(p);
  allocs_.clear();
  if (d_log_) cudaFree(d_log_);
  if (d_log_cursor_) cudaFree(d_log_cursor_);
  if (d_model_) cudaFree(d_model_);
  d_log_ = nullptr;
  d_log_cursor_ = nullptr;
  d_model_ = nullptr;
  log_cap_ = 0;
  if (stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
  if (stream2_) cudaStreamDestroy(stream2_);
  stream2_ = nullptr;
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  ev_fork_ = ev_join_ = nullptr;
  plastic_ = false;
  stdp_ = StdpArgs{};
  d_last_rev_ = nullptr;
  d_den_steps_ = nullptr;
  d_rev_ring_ = nullptr;
  d_rev_cnt_ = nullptr;
  rev_R_ = rev_cap_ = 0;
  pl_pos_.clear();
  pl_of_edge_.clear();
}

void Engine::invalidate_graphs() {
  for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
  graphs_.clear();
}

// propagator_32 of src/propagator_stability.cu:31-52 (double precision)
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

// ---------------------------------------------------------------------------
// Calibrate (src/nestgpu.cu:294-352 and the models' Calibrate methods)
// ---------------------------------------------------------------------------
void Engine::calibrate() {
  if (calibrated_) throw NgpuError("Calibration can be made only once");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw NgpuError("no CUDA device: the engine needs a GPU to calibrate and simulate");
  }
  if (verbosity >= 1) printf("Calibrating ...\n");
  calibrated_ = true;
  neural_time_ = 0.0;
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  cuda_check(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking), "stream");
  cuda_check(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming), "event");
  cuda_check(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming), "event");
  const int N = n_nodes();

  // ---- model-level calibration on the host parameter tables
  size_t acc_total = 0;
  for (auto &g : groups_) {
    if (is_aeif(g.model)) {
      const int npp = n_port_par(g.model);
      for (int i = 0; i < g.n; i++) {
        g.par[A_refractory_step][i] = 0.0f;
        for (int p = 0; p < g.nport; p++) {
          auto P = [&](int k) -> float & { return g.par[A_NSCAL + npp * p + k][i]; };
          if (g.model == M_AEIF_COND_BETA) {
            // g0 normalisation (src/aeif_cond_beta_multisynapse.cu:70-99)
            float td = P(2), tr = P(1);
            float denom1 = td - tr, denom2 = 0.0f;
            if (denom1 != 0.0f) {
              float t_p = td * tr * logf(td / tr) / denom1;
              denom2 = expf(-t_p / td) - expf(-t_p / tr);
            }
            if (denom2 == 0.0f) P(3) = (float)(M_E / td);
            else P(3) = (float)((1.0 / tr - 1.0 / td) / denom2);
          } else if (g.model == M_AEIF_COND_ALPHA) {
            P(2) = (float)(M_E / P(1));
          } else if (g.model == M_AEIF_PSC_ALPHA) {
            P(1) = (float)(M_E / P(0));
          }
        }
        if ((g.model == M_AEIF_PSC_EXP || g.model == M_AEIF_PSC_ALPHA) && g.par[A_Delta_T][i] <= 0.0f)
          g.par[A_V_peak][i] = g.par[A_V_th][i];
      }
    } else if (g.model == M_IAF_PSC_EXP) {
      for (int i = 0; i < g.n; i++) {
        // src/iaf_psc_exp.cu:68-82, propagators in double precision
        const double h = dt, tau_m = g.par[I_tau_m][i], C_m = g.par[I_C_m][i];
        const double tau_ex = g.par[I_tau_ex][i], tau_in = g.par[I_tau_in][i];
        float P22 = (float)std::exp(-h / tau_m);
        g.par[I_P11ex][i] = (float)std::exp(-h / tau_ex);
        g.par[I_P11in][i] = (float)std::exp(-h / tau_in);
        g.par[I_P22][i] = P22;
        g.par[I_P21ex][i] = (float)propagator_32(tau_ex, tau_m, C_m, h);
        g.par[I_P21in][i] = (float)propagator_32(tau_in, tau_m, C_m, h);
        g.par[I_P20][i] = (float)(tau_m / C_m * (1.0 - (double)P22));
      }
    }
    g.acc_off = acc_total;
    acc_total += (size_t)g.n * g.nport;
    g.dirty = true;
  }
  if (acc_total >= (1ULL << 32)) throw NgpuError("input accumulator exceeds 2^32 entries");
  n_acc_ = acc_total;

  // ---- partition: this process simulates neurons lo .. hi-1 of every group (a contiguous
  //      share per rank); the delivery layout keeps the in-edges of those neurons only
  std::vector<unsigned char> local(N, 1);
  for (auto &g : groups_) {
    g.lo = (int)((long long)g.n * part_rank_ / part_world_);
    g.hi = (int)((long long)g.n * (part_rank_ + 1) / part_world_);
    if (part_world_ > 1)
      for (int i = 0; i < g.n; i++) local[g.i0 + i] = (i >= g.lo && i < g.hi) ? 1 : 0;
  }
  // ---- connections: recurrent edges into CSR by (source, delay); poiss_gen edges apart
  const size_t E = c_src_.size();
  std::vector<unsigned char> is_pg(N, 0);
  for (auto &g : groups_)
    if (g.model == M_POISS_GEN)
      for (int i = 0; i < g.n; i++) is_pg[g.i0 + i] = 1;
  int dmin = INT32_MAX, dmax = INT32_MIN;
  size_t n_rec_edges = 0;
  for (size_t e = 0; e < E; e++) {
    Group &tg = groups_[node_group_[c_tgt_[e]]];
    if (c_port_[e] >= tg.nport)
      throw NgpuError("receptor port " + std::to_string(c_port_[e]) + " out of range for target node " +
                      std::to_string(c_tgt_[e]));
    if (is_pg[c_src_[e]]) {
      if (syn_of(e)) throw NgpuError("poiss_gen connections cannot be plastic");
      continue;
    }
    n_rec_edges++;
    if (syn_of(e)) plastic_ = true;
    dmin = std::min(dmin, c_d_[e]);
    dmax = std::max(dmax, c_d_[e]);
  }
  if (plastic_ && part_world_ > 1) throw NgpuError("a partitioned network cannot have plastic connections");
  std::vector<GenBlockDev> gblocks;
  for (size_t bi = 0; bi < blocks_.size(); bi++) {
    const GenBlock &b = blocks_[bi];
    Group &tg = group_of(b.tgt0);
    GenBlockDev d;
    d.src0 = b.src0;
    d.nsrc = b.nsrc;
    d.ntgt = b.ntgt;
    d.k = b.k;
    d.tgt_i0_rel = b.tgt0 - tg.i0;
    d.group_n = tg.n;
    d.acc_base = tg.acc_off + (unsigned long long)b.port * tg.n;
    d.w = b.w;
    d.dlo = (int)std::round(b.dmin_ms / dt) - 1;
    d.dhi = (int)std::round(b.dmax_ms / dt) - 1;
    d.seed = b.seed;
    // the block's targets simulated here (block-relative); the draws stay keyed by the
    // block-relative target, so every rank generates the same edges for a target
    const int loc_lo = tg.i0 + tg.lo, loc_hi = tg.i0 + tg.hi;
    d.t_begin = std::max(0, loc_lo - b.tgt0);
    d.t_end = std::min(b.ntgt, loc_hi - b.tgt0);
    if (d.t_end < d.t_begin) d.t_end = d.t_begin;
    dmin = std::min(dmin, d.dlo);
    dmax = std::max(dmax, d.dhi);
    gblocks.push_back(d);
  }
  // rule blocks expanded on the device: their delay steps, and target ports checked here
  // (the host path checks them edge by edge above)
  std::vector<RuleBlockDev> rdev;
  unsigned *d_node_acc0 = nullptr;
  int *d_node_gn = nullptr;
  if (!rblocks_.empty()) {
    for (const auto &b : rblocks_) {
      const RuleBlockDev &v = b.dev;
      for (int i = 0; i < v.nt; i++) {
        const int t = b.tgt_arr.empty() ? v.tgt0 + i : b.tgt_arr[i];
        if (v.port >= groups_[node_group_[t]].nport)
          throw NgpuError("receptor port " + std::to_string(v.port) + " out of range for target node " +
                          std::to_string(t));
      }
      dmin = std::min(dmin, b.dlo);
      dmax = std::max(dmax, b.dhi);
      rdev.push_back(v);
    }
    std::vector<unsigned> acc0(N, 0);
    std::vector<int> gn(N, 0);
    for (auto &g : groups_)
      for (int i = 0; i < g.n; i++) {
        acc0[g.i0 + i] = (unsigned)(g.acc_off + (size_t)i);
        gn[g.i0 + i] = g.n;
      }
    // non-local targets get the index 0xffffffff: the expansion skips them
    if (part_world_ > 1)
      for (int i = 0; i < N; i++)
        if (!local[i]) acc0[i] = 0xffffffffu;
    d_node_acc0 = dalloc<unsigned>(N);
    d_node_gn = dalloc<int>(N);
    cuda_check(cudaMemcpy(d_node_acc0, acc0.data(), N * sizeof(unsigned), cudaMemcpyHostToDevice), "node map");
    cuda_check(cudaMemcpy(d_node_gn, gn.data(), N * sizeof(int), cudaMemcpyHostToDevice), "node map");
  }
  if (n_rec_edges == 0 && gblocks.empty() && rdev.empty()) { dmin = 0; dmax = 0; }
  dmin_ = dmin;
  dspan_ = dmax - dmin + 1;
  if (dspan_ > deliver_max_pairs())
    throw NgpuError("delay range exceeds " + std::to_string(deliver_max_pairs()) + " time steps");
  d_has_out_ = dalloc<unsigned char>(N);
  std::vector<size_t> pl_edge;       // plastic host edges with their (source, delay) key and rank
  std::vector<long long> pl_key;
  std::vector<int> pl_rank;
  {
    // host edges: per-key counts and each edge's rank inside its (source, delay) segment,
    // in insertion order; the device does the scan, placement and generated blocks
    const size_t nkey = (size_t)N * dspan_;
    std::vector<int> cnt;
    std::vector<long long> hkey;
    std::vector<int> hrank;
    std::vector<EdgeW> hew;
    pl_edge.clear();
    pl_key.clear();
    pl_rank.clear();
    if (n_rec_edges) {
      cnt.assign(nkey, 0);
      hkey.reserve(n_rec_edges);
      hrank.reserve(n_rec_edges);
      hew.reserve(n_rec_edges);
      for (size_t e = 0; e < E; e++) {
        if (is_pg[c_src_[e]] || !local[c_tgt_[e]]) continue;
        const Group &tg = groups_[node_group_[c_tgt_[e]]];
        long long key = (long long)c_src_[e] * dspan_ + (c_d_[e] - dmin);
        if (syn_of(e)) {
          pl_edge.push_back(e);
          pl_key.push_back(key);
          pl_rank.push_back(cnt[key]);
        }
        hkey.push_back(key);
        hrank.push_back(cnt[key]++);
        EdgeW x;
        x.acc = (uint32_t)(tg.acc_off + (size_t)c_port_[e] * tg.n + (c_tgt_[e] - tg.i0));
        x.w = c_w_[e];
        hew.push_back(x);
      }
    }
    unsigned long long *d_off = nullptr;
    EdgeW *d_edge = nullptr;
    size_t n_edge = 0;
    build_csr_device(N, dmin_, dspan_, cnt, hkey, hrank, hew, gblocks, rdev, d_node_acc0, d_node_gn, &d_off,
                     &d_edge, &n_edge, d_has_out_, stream_);
    allocs_.push_back(d_off);
    allocs_.push_back(d_edge);
    d_ev_off_ = (long long *)d_off;
    d_edge_ = d_edge;
    n_edge_dev_ = n_edge;
  }
  std::vector<unsigned char> has_out(N, 0);
  cuda_check(cudaMemcpy(has_out.data(), d_has_out_, N, cudaMemcpyDeviceToHost), "has_out");
  int n_src_out = 0;
  for (int i = 0; i < N; i++) n_src_out += has_out[i];
  d_has_out_all_ = nullptr;
  if (part_world_ > 1) {
    // sources with recurrent edges to any process's neurons: their spikes are exchanged
    std::vector<unsigned char> all(N, 0);
    for (size_t e = 0; e < E; e++)
      if (!is_pg[c_src_[e]]) all[c_src_[e]] = 1;
    d_has_out_all_ = dalloc<unsigned char>(N);
    cuda_check(cudaMemcpy(d_has_out_all_, all.data(), N, cudaMemcpyHostToDevice), "has_out_all");
    mark_sources_device(gblocks, rdev, d_has_out_all_, stream_);
    cuda_check(cudaStreamSynchronize(stream_), "has_out_all");
  }

  // ---- poiss_gen: generator table and target-major in-edges with canonical ids
  n_gen_ = 0;
  for (auto &g : groups_)
    if (g.model == M_POISS_GEN) { g.gen0 = n_gen_; n_gen_ += g.n; }
  d_gen_ = dalloc<GenPar>(n_gen_);
  {
    struct DE { int tgt; PoissonIn pe; };
    std::vector<DE> de;
    // the generators' out-edges in reference order: source-major, delay groups ascending,
    // insertion order (src/connect.cu:38-74)
    std::vector<long long> pg_edges;
    for (size_t e = 0; e < E; e++)
      if (is_pg[c_src_[e]]) pg_edges.push_back((long long)e);
    std::stable_sort(pg_edges.begin(), pg_edges.end(), [&](long long a, long long b) {
      return c_src_[a] != c_src_[b] ? c_src_[a] < c_src_[b] : c_d_[a] < c_d_[b];
    });
    size_t q = 0;
    for (int s = 0; s < N; s++) {
      if (!is_pg[s]) continue;
      const Group &pg = groups_[node_group_[s]];
      const int gi = pg.gen0 + (s - pg.i0);
      const uint32_t set = pg.pg_stream.empty() ? 0xffffffffu : pg.pg_stream[s - pg.i0];
      const uint32_t stream = set == 0xffffffffu ? (uint32_t)gi : set;
      uint32_t id = 0;   // out-edges of this generator in connection order
      for (; q < pg_edges.size() && c_src_[pg_edges[q]] == s; q++) {
        long long e = pg_edges[q];
        DE x;
        x.tgt = c_tgt_[e];
        x.pe.edge_id = id++;
        x.pe.gen = gi;
        x.pe.weight = c_w_[e];
        x.pe.delay = dt * (float)(c_d_[e] + 1);
        x.pe.port = c_port_[e];
        x.pe.stream = stream;
        de.push_back(x);
      }
    }
    std::stable_sort(de.begin(), de.end(), [](const DE &a, const DE &b) { return a.tgt < b.tgt; });
    size_t k = 0;
    for (auto &g : groups_) {
      if (g.nport == 0) continue;
      std::vector<int> off(g.n + 1, 0);
      std::vector<PoissonIn> pin;
      while (k < de.size() && de[k].tgt < g.i0) k++;
      size_t k0 = k;
      while (k < de.size() && de[k].tgt < g.i0 + g.n) {
        off[de[k].tgt - g.i0 + 1]++;
        pin.push_back(de[k].pe);
        k++;
      }
      (void)k0;
      if (pin.empty()) continue;
      for (int i = 0; i < g.n; i++) off[i + 1] += off[i];
      g.d_pin_off = dalloc<int>(g.n + 1);
      g.d_pin = dalloc<PoissonIn>(pin.size());
      cuda_check(cudaMemcpy(g.d_pin_off, off.data(), (g.n + 1) * sizeof(int), cudaMemcpyHostToDevice), "pin_off");
      cuda_check(cudaMemcpy(g.d_pin, pin.data(), pin.size() * sizeof(PoissonIn), cudaMemcpyHostToDevice), "pin");
    }
  }

  // ---- time batching: M steps per batch, M <= min delay in steps (spikes emitted inside
  //      a batch arrive after it); one accumulator slot per step of a batch
  batch_ = (n_rec_edges || !gblocks.empty() || !rdev.empty()) ? std::min(dmin_ + 1, MAX_BATCH) : MAX_BATCH;
  batch_ = std::max(1, std::min(batch_, batch_max));
  // plastic edges: one step per batch, so that each step's weight changes see the post-
  // synaptic spikes of the same step (src/nestgpu.cu:469-635 order)
  if (plastic_) batch_ = 1;
  if (dspan_ * batch_ > deliver_max_pairs()) batch_ = std::max(1, deliver_max_pairs() / dspan_);
  d_acc_ = dalloc<double>(n_acc_ * batch_);
  cuda_check(cudaMemset(d_acc_, 0, std::max<size_t>(n_acc_ * batch_, 1) * sizeof(double)), "memset");
  // delivery at emission: a spike of step t reaches steps t + 1 + dmin .. t + dmin + dspan,
  // all after its batch (batch_ <= dmin + 1); the ring has one slot per step of that reach
  // and of the batch being read, so a slot being read is never one being written
  push_ = deliver_push && push_eligible();
  push_R_ = 0;
  d_pacc_ = nullptr;
  if (push_) {
    push_R_ = batch_ + dmin_ + dspan_;
    d_pacc_ = dalloc<double>(n_acc_ * (size_t)push_R_);
    cuda_check(cudaMemset(d_pacc_, 0, std::max<size_t>(n_acc_ * (size_t)push_R_, 1) * sizeof(double)), "memset");
  }

  // ---- spike ring and per-node spike state
  R_ = (dmin_ + dspan_ - 1) + batch_ + 3;
  cap_ = (int)std::min<long long>((long long)n_src_out * std::max(1.0f, max_spike_num_fact) + 1024, 1LL << 30);
  d_ring_ = dalloc<int2>((size_t)R_ * cap_);
  d_ring_cnt_ = dalloc<int>(R_);
  cuda_check(cudaMemset(d_ring_cnt_, 0, R_ * sizeof(int)), "ring_cnt");
  d_last_tidx_ = dalloc<int>(N);
  cuda_check(cudaMemset(d_last_tidx_, 0xff, (size_t)N * sizeof(int)), "last_tidx");
  d_last_h_ = dalloc<float>(N);
  cuda_check(cudaMemset(d_last_h_, 0, (size_t)N * sizeof(float)), "last_h");
  d_status_ = dalloc<unsigned>(1);
  cuda_check(cudaMemset(d_status_, 0, sizeof(unsigned)), "status");
  d_counters_ = dalloc<unsigned long long>(4);
  cuda_check(cudaMemset(d_counters_, 0, 4 * sizeof(unsigned long long)), "counters");
  d_clk_ = dalloc<Clock>(1);
  cuda_check(cudaMemset(d_clk_, 0, sizeof(Clock)), "clock");
  deliver_blocks_ = std::max(1, std::min(148 * 8, (n_src_out + 63) / 64));
  if (plastic_) build_plastic(pl_edge, pl_key, pl_rank);
  // ---- dendritic delays: the reverse ring (plastic networks only; src/spike_buffer.cu:162-317)
  if (plastic_) {
    std::vector<int> den(N, 0);
    int dmax_den = 0;
    for (auto &g : groups_) {
      int pi = -1;
      if (is_aeif(g.model)) pi = A_den_delay;
      else if (g.model == M_IAF_PSC_EXP) pi = I_den_delay;
      else if (g.model == M_PARROT) pi = 1;
      if (pi < 0) continue;
      for (int i = 0; i < g.n; i++) {
        // round(den_delay / dt) in float, as src/spike_buffer.cu:175-177
        const int d = (int)std::round(g.par[pi][i] / dt);
        if (d < 0) throw NgpuError("dendritic delay must be >= 0");
        den[g.i0 + i] = d;
        dmax_den = std::max(dmax_den, d);
      }
    }
    d_last_rev_ = dalloc<int>(N);
    cuda_check(cudaMemset(d_last_rev_, 0xff, (size_t)N * sizeof(int)), "last_rev");
    stdp_.last_tidx = d_last_rev_;
    if (dmax_den > 0) {
      d_den_steps_ = dalloc<int>(N);
      cuda_check(cudaMemcpy(d_den_steps_, den.data(), N * sizeof(int), cudaMemcpyHostToDevice), "den_delay");
      rev_R_ = dmax_den + 2;
      rev_cap_ = N;
      d_rev_ring_ = dalloc<int>((size_t)rev_R_ * rev_cap_);
      d_rev_cnt_ = dalloc<int>(rev_R_);
      cuda_check(cudaMemset(d_rev_cnt_, 0, rev_R_ * sizeof(int)), "rev_cnt");
    }
  }

  // ---- per-group device state
  for (auto &g : groups_) {
    if (is_aeif(g.model) || g.model == M_IAF_PSC_EXP || g.model == M_PARROT || g.model == M_SPIKE_DET) {
      const int nvar = (int)g.var.size();
      g.d_var = dalloc<float>((size_t)nvar * g.n);
      for (int v = 0; v < nvar; v++)
        cuda_check(cudaMemcpy(g.d_var + (size_t)v * g.n, g.var[v].data(), g.n * sizeof(float),
                              cudaMemcpyHostToDevice), "var");
    }
    if (is_aeif(g.model)) {
      g.d_strag = dalloc<int2>(g.n);
      g.strag_slot = n_strag_++;
      g.d_refr = dalloc<float>(g.n);
      cuda_check(cudaMemcpy(g.d_refr, g.par[A_refractory_step].data(), g.n * sizeof(float),
                            cudaMemcpyHostToDevice), "refr");
      std::vector<double> x(g.n, 0.0);
      std::vector<float> h(g.n, g.h0_rel * dt);
      g.d_x = dalloc<double>(g.n);
      g.d_h = dalloc<float>(g.n);
      cuda_check(cudaMemcpy(g.d_x, x.data(), g.n * sizeof(double), cudaMemcpyHostToDevice), "x");
      cuda_check(cudaMemcpy(g.d_h, h.data(), g.n * sizeof(float), cudaMemcpyHostToDevice), "h");
    }
    if (g.model == M_PARROT || g.model == M_SPIKE_DET) {
      g.d_hold = dalloc<float>(g.n);
      cuda_check(cudaMemcpy(g.d_hold, g.par[0].data(), g.n * sizeof(float), cudaMemcpyHostToDevice), "hold");
    }
    if (g.spike_count_on) {
      g.d_spike_count = dalloc<int>(g.n);
      cuda_check(cudaMemset(g.d_spike_count, 0, g.n * sizeof(int)), "spike_count");
    }
    if (g.max_rec > 0) {
      g.d_n_rec = dalloc<int>(g.n);
      g.d_rec_times = dalloc<float>((size_t)g.n * g.max_rec);
      cuda_check(cudaMemset(g.d_n_rec, 0, g.n * sizeof(int)), "n_rec");
    }
    if (g.model == M_SPIKE_GEN) {
      // src/spike_generator.cu:230-290: time indices round((t - t_min)/dt), strictly increasing
      std::vector<int> off(g.n + 1, 0), tix;
      std::vector<float> hh;
      for (int i = 0; i < g.n; i++) {
        const auto &t = g.sg_times[i];
        std::vector<float> hs = g.sg_heights[i];
        if (!t.empty()) {
          if (hs.empty()) hs.assign(t.size(), 1.0f);
          else if (hs.size() != t.size())
            throw NgpuError("spike time array and spike height array must have the same size in spike generator");
        }
        for (size_t k = 0; k < t.size(); k++) {
          int ti = (int)std::round((t[k] - 0.0f) / dt);
          if (k > 0 && ti <= tix.back())
            throw NgpuError("Spike times must be ordered, and the difference between\nconsecutive spikes must be >= the time resolution");
          tix.push_back(ti);
          hh.push_back(hs[k]);
        }
        off[i + 1] = (int)tix.size();
      }
      g.d_sg_off = dalloc<int>(g.n + 1);
      g.d_sg_tidx = dalloc<int>(tix.size());
      g.d_sg_h = dalloc<float>(hh.size());
      g.d_sg_next = dalloc<int>(g.n);
      cuda_check(cudaMemcpy(g.d_sg_off, off.data(), (g.n + 1) * sizeof(int), cudaMemcpyHostToDevice), "sg");
      if (!tix.empty()) {
        cuda_check(cudaMemcpy(g.d_sg_tidx, tix.data(), tix.size() * sizeof(int), cudaMemcpyHostToDevice), "sg");
        cuda_check(cudaMemcpy(g.d_sg_h, hh.data(), hh.size() * sizeof(float), cudaMemcpyHostToDevice), "sg");
      }
      cuda_check(cudaMemset(g.d_sg_next, 0, g.n * sizeof(int)), "sg");
    }
  }
  d_strag_cnt_ = dalloc<int>(std::max(1, n_strag_));
  cuda_check(cudaMemset(d_strag_cnt_, 0, std::max(1, n_strag_) * sizeof(int)), "strag");
  build_records();
  cuda_check(cudaDeviceSynchronize(), "calibrate");
}

// Derived parameters: uniform over the group -> kernel argument, else device array.
void Engine::upload_params() {
  bool any = false;
  // device arrays of the previous upload, reused when a parameter stays non-uniform (a
  // step loop that sets parameters between steps allocates nothing after the first change)
  std::vector<float *> prev;
  auto put = [&](Group &g, int slot, const std::vector<float> &v) {
    bool uni = true;
    for (int i = 1; i < g.n && uni; i++) uni = (std::memcmp(&v[i], &v[0], 4) == 0);
    if (uni) {
      g.der_val[slot] = v[0];
      g.d_der[slot] = nullptr;
    } else {
      float *d = (slot < (int)prev.size() && prev[slot]) ? prev[slot] : dalloc<float>(g.n);
      cuda_check(cudaMemcpy(d, v.data(), g.n * sizeof(float), cudaMemcpyHostToDevice), "param");
      g.der_val[slot] = 0.0f;
      g.d_der[slot] = d;
    }
  };
  std::vector<GenPar> gp(n_gen_);
  bool gen_dirty = false;
  for (auto &g : groups_) {
    if (!g.dirty) continue;
    // aeif and iaf parameters can travel as kernel arguments, baked into the captured graphs;
    // poiss_gen and parrot parameters live in device tables that the kernels read each step
    if (is_aeif(g.model) || g.model == M_IAF_PSC_EXP) any = true;
    g.dirty = false;
    const int n = g.n;
    std::vector<float> v(n);
    if ((g.model == M_PARROT || g.model == M_SPIKE_DET) && g.d_hold)
      cuda_check(cudaMemcpy(g.d_hold, g.par[0].data(), n * sizeof(float), cudaMemcpyHostToDevice), "hold");
    prev = g.d_der;
    if (is_aeif(g.model)) {
      g.der_val.assign(AEIF_NPAR, 0.0f);
      g.d_der.assign(AEIF_NPAR, nullptr);
      auto cp = [&](int slot, int src) { put(g, slot, g.par[src]); };
      cp(AP_V_th, A_V_th);
      cp(AP_Delta_T, A_Delta_T);
      for (int i = 0; i < n; i++) v[i] = 1.0f / g.par[A_Delta_T][i];
      put(g, AP_inv_Delta_T, v);
      cp(AP_g_L, A_g_L);
      cp(AP_E_L, A_E_L);
      for (int i = 0; i < n; i++) v[i] = 1.0f / g.par[A_C_m][i];
      put(g, AP_inv_C_m, v);
      cp(AP_a, A_a);
      cp(AP_b, A_b);
      for (int i = 0; i < n; i++) v[i] = 1.0f / g.par[A_tau_w][i];
      put(g, AP_inv_tau_w, v);
      cp(AP_I_e, A_I_e);
      cp(AP_V_peak, A_V_peak);
      cp(AP_V_reset, A_V_reset);
      for (int i = 0; i < n; i++) {
        float rs = (float)(int)roundf(g.par[A_t_ref][i] / dt);
        v[i] = rs < 0.0f ? 0.0f : rs;
      }
      put(g, AP_refr_steps, v);
      const int npp = n_port_par(g.model);
      for (int p = 0; p < g.nport; p++) {
        const int b = AEIF_NSCAL + AEIF_NPORTPAR * p, hb = A_NSCAL + npp * p;
        std::vector<float> er(n, 0.0f), t1(n), t2(n), pw(n, 1.0f);
        for (int i = 0; i < n; i++) {
          switch (g.model) {
          case M_AEIF_COND_BETA:
            er[i] = g.par[hb + 0][i]; t1[i] = 1.0f / g.par[hb + 1][i]; t2[i] = 1.0f / g.par[hb + 2][i];
            pw[i] = g.par[hb + 3][i];
            break;
          case M_AEIF_COND_ALPHA:
            er[i] = g.par[hb + 0][i]; t1[i] = 1.0f / g.par[hb + 1][i]; t2[i] = t1[i]; pw[i] = g.par[hb + 2][i];
            break;
          case M_AEIF_PSC_EXP:
            t1[i] = 1.0f / g.par[hb + 0][i]; t2[i] = t1[i];
            break;
          default:
            t1[i] = 1.0f / g.par[hb + 0][i]; t2[i] = t1[i]; pw[i] = g.par[hb + 1][i];
            break;
          }
        }
        put(g, b + 0, er);
        put(g, b + 1, t1);
        put(g, b + 2, t2);
        put(g, b + 3, pw);
      }
    } else if (g.model == M_IAF_PSC_EXP) {
      g.der_val.assign(IP_NPAR, 0.0f);
      g.d_der.assign(IP_NPAR, nullptr);
      put(g, IP_I_e, g.par[I_I_e]);
      put(g, IP_Theta_rel, g.par[I_Theta_rel]);
      put(g, IP_V_reset_rel, g.par[I_V_reset_rel]);
      for (int i = 0; i < n; i++) v[i] = (float)(int)roundf(g.par[I_t_ref][i] / dt);
      put(g, IP_refr_steps, v);
      put(g, IP_P20, g.par[I_P20]);
      put(g, IP_P11ex, g.par[I_P11ex]);
      put(g, IP_P11in, g.par[I_P11in]);
      put(g, IP_P21ex, g.par[I_P21ex]);
      put(g, IP_P21in, g.par[I_P21in]);
      put(g, IP_P22, g.par[I_P22]);
    } else if (g.model == M_POISS_GEN) {
      gen_dirty = true;
    }
  }
  if (gen_dirty && n_gen_ > 0) {
    for (auto &g : groups_) {
      if (g.model != M_POISS_GEN) continue;
      for (int i = 0; i < g.n; i++)
        gp[g.gen0 + i] = {g.par[PG_rate][i], g.par[PG_origin][i], g.par[PG_start][i], g.par[PG_stop][i]};
    }
    cuda_check(cudaMemcpy(d_gen_, gp.data(), n_gen_ * sizeof(GenPar), cudaMemcpyHostToDevice), "gen");
  }
  if (any) invalidate_graphs();
}

// Record columns: per group a CSR over its neurons of {variable code, column}; the
// update kernels write them into a [rows][ncol] window buffer, the host adds the time.
void Engine::build_records() {
  rec_ncol_ = 0;
  std::vector<std::vector<std::vector<int2>>> per(groups_.size());
  for (size_t r = 0; r < records_.size(); r++) {
    RecordSpec &rs = records_[r];
    for (size_t c = 0; c < rs.var.size(); c++) {
      const int gi = group_index(rs.node[c]);
      Group &g = groups_[gi];
      const int rel = rs.node[c] - g.i0;
      int code = -1;
      if (rs.var[c] != "spike") {
        int idx;
        Kind k = locate(rs.node[c], rs.var[c], &idx);
        if (is_aeif(g.model)) {
          const int nvar = 2 + n_port_var(g.model) * g.nport;
          if (k == K_SCAL_VAR) code = idx;
          else if (k == K_PORT_VAR) code = 2 + n_port_var(g.model) * rs.port[c] + idx;
          else code = nvar;   // refractory counter
        } else {
          code = idx;
        }
      }
      if (per[gi].empty()) per[gi].resize(g.n);
      per[gi][rel].push_back(make_int2(code, rec_ncol_));
      rec_ncol_++;
    }
    if (!rs.file.empty()) {
      rs.fp = fopen(rs.file.c_str(), "w");
      if (!rs.fp) throw NgpuError("cannot open record file " + rs.file);
    }
  }
  for (size_t gi = 0; gi < groups_.size(); gi++) {
    if (per[gi].empty()) continue;
    Group &g = groups_[gi];
    std::vector<int> first(g.n + 1, 0);
    std::vector<int2> cols;
    for (int i = 0; i < g.n; i++) {
      first[i] = (int)cols.size();
      cols.insert(cols.end(), per[gi][i].begin(), per[gi][i].end());
    }
    first[g.n] = (int)cols.size();
    g.d_rec_first = dalloc<int>(g.n + 1);
    g.d_rec_col = dalloc<int2>(cols.size());
    cuda_check(cudaMemcpy(g.d_rec_first, first.data(), (g.n + 1) * sizeof(int), cudaMemcpyHostToDevice), "rec");
    cuda_check(cudaMemcpy(g.d_rec_col, cols.data(), cols.size() * sizeof(int2), cudaMemcpyHostToDevice), "rec");
  }
}

// ---------------------------------------------------------------------------
// Kernel argument blocks
// ---------------------------------------------------------------------------
SpikeOut Engine::spike_out() const {
  SpikeOut so;
  so.ring = d_ring_;
  so.ring_cnt = d_ring_cnt_;
  so.R = R_;
  so.cap = cap_;
  so.has_out = d_has_out_;
  so.has_out_all = d_has_out_all_ ? d_has_out_all_ : d_has_out_;
  so.xch = part_world_ > 1 ? xch_send_ : nullptr;
  so.xch_cap = xch_cap_;
  so.last_tidx = d_last_tidx_;
  so.last_height = d_last_h_;
  so.status = d_status_;
  so.n_spikes = d_counters_ + 2;
  so.last_rev = d_last_rev_;
  so.den_steps = d_den_steps_;
  so.rev_ring = d_rev_ring_;
  so.rev_cnt = d_rev_cnt_;
  so.rev_R = rev_R_;
  so.rev_cap = rev_cap_;
  return so;
}

PushOut Engine::push_out() const {
  PushOut po;
  po.acc = d_pacc_;
  po.R = push_R_;
  po.stride = n_acc_;
  po.ev_off = d_ev_off_;
  po.edge = d_edge_;
  po.dmin = dmin_;
  po.dspan = dspan_;
  po.n_events = d_counters_ + 1;
  return po;
}

static GroupSpikeRec spike_rec(Group &g) {
  GroupSpikeRec r;
  r.spike_count = g.d_spike_count;
  r.n_rec = g.d_n_rec;
  r.rec_times = g.d_rec_times;
  r.max_rec = g.max_rec;
  return r;
}

GroupRecord Engine::group_record(Group &g) {
  GroupRecord r;
  r.first = g.d_rec_first;
  r.col = g.d_rec_col;
  r.buf = d_recbuf_;
  r.ncol = rec_ncol_;
  if (!d_recbuf_) r.first = nullptr;
  return r;
}

GroupInput Engine::group_input(Group &g) {
  GroupInput in;
  in.acc = d_acc_ + g.acc_off;
  in.slot_stride = n_acc_;
  if (push_ && g.model == M_IAF_PSC_EXP) in.acc = d_pacc_ + g.acc_off;   // the delivery-at-emission ring
  in.pin_off = g.d_pin_off;
  in.pin = g.d_pin;
  in.gen = d_gen_;
  in.lam_scale = (float)(dt / 1000.0);
  in.seed = kernel_seed;
  return in;
}

AeifArgs Engine::aeif_args(Group &g) {
  AeifArgs A;
  std::memset(&A, 0, sizeof(A));
  A.n = g.n;
  A.i0 = g.i0;
  A.lo = g.lo;
  A.hi = g.hi;
  A.nport = g.nport;
  A.nvar = 2 + n_port_var(g.model) * g.nport;
  A.var = g.d_var;
  A.refr = g.d_refr;
  A.x = g.d_x;
  A.h = g.d_h;
  A.in = group_input(g);
  A.rec = group_record(g);
  A.dt = dt;
  A.hmin = g.h_min_rel * dt;
  A.hmin_acc = A.hmin * 1.00001f;
  A.nderiv = d_counters_;
  A.budget = rk5_budget > 0 ? batch_ + rk5_budget : 0;
  A.strag_list = g.d_strag;
  A.strag_cnt = d_strag_cnt_ + g.strag_slot;
  A.srec = spike_rec(g);
  A.threads = update_threads;
  A.occupancy = update_occupancy;
  A.trial_iter = update_trial_iter;
  A.uniform = 1;
  for (int j = 0; j < AEIF_NSCAL + AEIF_NPORTPAR * g.nport && j < AEIF_NPAR; j++)
    if (g.d_der[j]) A.uniform = 0;
  A.learn.mode = learn_mode_;
  A.learn.log = d_log_;
  A.learn.log_cursor = d_log_cursor_;
  A.learn.log_cap = (unsigned long long)log_cap_;
  A.learn.model = d_model_;
  for (int j = 0; j < AEIF_NPAR; j++) {
    A.pval[j] = g.der_val[j];
    A.parr[j] = g.d_der[j];
  }
  return A;
}

IafArgs Engine::iaf_args(Group &g) {
  IafArgs A;
  std::memset(&A, 0, sizeof(A));
  A.n = g.n;
  A.i0 = g.i0;
  A.lo = g.lo;
  A.hi = g.hi;
  A.var = g.d_var;
  A.in = group_input(g);
  A.rec = group_record(g);
  A.dt = dt;
  A.srec = spike_rec(g);
  for (int j = 0; j < IP_NPAR; j++) {
    A.pval[j] = g.der_val[j];
    A.parr[j] = g.d_der[j];
  }
  return A;
}

ParrotArgs Engine::parrot_args(Group &g) {
  ParrotArgs A;
  A.n = g.n;
  A.i0 = g.i0;
  A.lo = g.lo;
  A.hi = g.hi;
  A.var = g.d_var;
  A.hold = g.d_hold;
  A.in = group_input(g);
  A.rec = group_record(g);
  A.dt = dt;
  A.srec = spike_rec(g);
  return A;
}

SpikeGenArgs Engine::sg_args(Group &g) {
  SpikeGenArgs A;
  A.n = g.n;
  A.i0 = g.i0;
  A.lo = g.lo;
  A.hi = g.hi;
  A.off = g.d_sg_off;
  A.tidx = g.d_sg_tidx;
  A.height = g.d_sg_h;
  A.next = g.d_sg_next;
  A.rec = group_record(g);
  A.dt = dt;
  A.srec = spike_rec(g);
  return A;
}

DeliverArgs Engine::deliver_args() {
  DeliverArgs A;
  A.ring = d_ring_;
  A.ring_cnt = d_ring_cnt_;
  A.R = R_;
  A.cap = cap_;
  A.dmin = dmin_;
  A.dspan = dspan_;
  A.ev_off = d_ev_off_;
  A.edge = d_edge_;
  A.acc = d_acc_;
  A.slot_stride = n_acc_;
  A.dt = dt;
  A.n_events = d_counters_ + 1;
  A.strag_cnt = d_strag_cnt_;
  A.n_strag = n_strag_;
  A.aggregate = deliver_aggregate;
  A.prefetch = deliver_prefetch;
  A.xch = part_world_ > 1 ? xch_send_ : nullptr;
  return A;
}

// ---------------------------------------------------------------------------
// Plastic edges: forward index over the delivery CSR's (source, delay) segments, reverse
// index by target (src/spike_buffer.cu:430-520), 16-bit arrival stamps starting at 0x8000
// (src/rev_spike.cu:150-155), synapse-group parameter table (src/syn_model.cu:170-238).
// ---------------------------------------------------------------------------
// Current weight of plastic host edge e (its device copy).
float Engine::plastic_weight(size_t e, float fallback) {
  auto it = std::lower_bound(pl_of_edge_.begin(), pl_of_edge_.end(), std::make_pair(e, INT32_MIN));
  if (it == pl_of_edge_.end() || it->first != e) return fallback;
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  EdgeW x;
  cuda_check(cudaMemcpy(&x, d_edge_ + pl_pos_[it->second], sizeof(EdgeW), cudaMemcpyDeviceToHost),
             "plastic weight");
  return x.w;
}

void Engine::upload_syn_groups() {
  const int ng = (int)syn_groups_.size();
  std::vector<int> type(ng);
  std::vector<float> par((size_t)ng * SYN_NPAR, 0.0f);
  for (int g = 0; g < ng; g++) {
    type[g] = syn_groups_[g].type;
    for (size_t k = 0; k < syn_groups_[g].par.size(); k++) par[(size_t)g * SYN_NPAR + k] = syn_groups_[g].par[k];
  }
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  cuda_check(cudaMemcpy((void *)stdp_.syn_type, type.data(), ng * sizeof(int), cudaMemcpyHostToDevice), "syn groups");
  cuda_check(cudaMemcpy((void *)stdp_.syn_par, par.data(), par.size() * sizeof(float), cudaMemcpyHostToDevice),
             "syn groups");
}

void Engine::build_plastic(const std::vector<size_t> &pl_edge, const std::vector<long long> &pl_key,
                           const std::vector<int> &pl_rank) {
  const int N = n_nodes();
  const size_t nkey = (size_t)N * dspan_;
  const size_t P = pl_edge.size();
  if (P >= (size_t)INT32_MAX) throw NgpuError("too many plastic connections");
  // a host edge sits at its segment's start plus its rank in the segment
  std::vector<unsigned long long> off(nkey + 1);
  cuda_check(cudaMemcpy(off.data(), d_ev_off_, (nkey + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
             "segment offsets");
  std::vector<size_t> ord(P);
  std::iota(ord.begin(), ord.end(), (size_t)0);
  std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
    return pl_key[a] != pl_key[b] ? pl_key[a] < pl_key[b] : pl_rank[a] < pl_rank[b];
  });
  std::vector<int> pl_off(nkey + 1, 0);
  std::vector<PlasticEdge> pl(P);
  pl_pos_.assign(P, 0);
  pl_of_edge_.resize(P);
  std::vector<int> cnt_t(N, 0);
  for (size_t q = 0; q < P; q++) {
    const size_t i = ord[q];
    pl_off[pl_key[i] + 1]++;
    PlasticEdge x;
    x.pos = off[pl_key[i]] + (unsigned long long)pl_rank[i];
    x.target = c_tgt_[pl_edge[i]];
    x.group = c_syn_[pl_edge[i]];
    pl[q] = x;
    pl_pos_[q] = x.pos;
    pl_of_edge_[q] = {pl_edge[i], (int)q};
    cnt_t[x.target]++;
  }
  for (size_t k = 0; k < nkey; k++) pl_off[k + 1] += pl_off[k];
  std::sort(pl_of_edge_.begin(), pl_of_edge_.end());
  // reverse index: targets with plastic in-edges, their entries in forward order
  std::vector<int> rev_node, rev_off{0}, first(N, -1);
  for (int t = 0; t < N; t++)
    if (cnt_t[t]) {
      first[t] = rev_off.back();
      rev_node.push_back(t);
      rev_off.push_back(rev_off.back() + cnt_t[t]);
    }
  std::vector<int> rev_id(P);
  for (size_t q = 0; q < P; q++) rev_id[first[pl[q].target]++] = (int)q;
  std::vector<unsigned short> stamp(P, 0x8000);

  StdpArgs &A = stdp_;
  int *d_pl_off = dalloc<int>(nkey + 1);
  PlasticEdge *d_pl = dalloc<PlasticEdge>(P);
  unsigned short *d_stamp = dalloc<unsigned short>(P);
  int *d_rev_off = dalloc<int>(rev_off.size());
  int *d_rev_id = dalloc<int>(P);
  int *d_rev_node = dalloc<int>(std::max<size_t>(rev_node.size(), 1));
  int *d_type = dalloc<int>(syn_groups_.size());
  float *d_par = dalloc<float>(syn_groups_.size() * SYN_NPAR);
  cuda_check(cudaMemcpy(d_pl_off, pl_off.data(), pl_off.size() * sizeof(int), cudaMemcpyHostToDevice), "stdp");
  cuda_check(cudaMemcpy(d_pl, pl.data(), P * sizeof(PlasticEdge), cudaMemcpyHostToDevice), "stdp");
  cuda_check(cudaMemcpy(d_stamp, stamp.data(), P * sizeof(unsigned short), cudaMemcpyHostToDevice), "stdp");
  cuda_check(cudaMemcpy(d_rev_off, rev_off.data(), rev_off.size() * sizeof(int), cudaMemcpyHostToDevice), "stdp");
  cuda_check(cudaMemcpy(d_rev_id, rev_id.data(), P * sizeof(int), cudaMemcpyHostToDevice), "stdp");
  if (!rev_node.empty())
    cuda_check(cudaMemcpy(d_rev_node, rev_node.data(), rev_node.size() * sizeof(int), cudaMemcpyHostToDevice),
               "stdp");
  A.ring = d_ring_;
  A.ring_cnt = d_ring_cnt_;
  A.R = R_;
  A.cap = cap_;
  A.dmin = dmin_;
  A.dspan = dspan_;
  A.pl_off = d_pl_off;
  A.pl = d_pl;
  A.stamp = d_stamp;
  A.n_pl = (long long)P;
  A.edge = d_edge_;
  A.last_tidx = d_last_tidx_;
  A.syn_type = d_type;
  A.syn_par = d_par;
  A.rev_off = d_rev_off;
  A.rev_id = d_rev_id;
  A.rev_node = d_rev_node;
  A.n_rev_nodes = (int)rev_node.size();
  A.dt = dt;
  upload_syn_groups();
}

// ---------------------------------------------------------------------------
// Step loop
// ---------------------------------------------------------------------------
// One batch of M steps starting at graph step k0: delivery, then every group.
void Engine::launch_batch(int k0, int M, std::vector<cudaEvent_t> *ev) {
  SpikeOut so = spike_out();
  const PushOut po = push_out();
  // With aeif groups and other spiking groups in the network, the others run on a second
  // stream next to the aeif kernels: they then fill the SMs that the aeif straggler tail
  // leaves idle.  The groups touch disjoint state (their own accumulator rows, node
  // entries and record columns; the spike ring only through atomics).
  bool has_aeif = false, has_other = false;
  for (auto &g : groups_) {
    if (g.n <= 0) continue;
    if (is_aeif(g.model)) has_aeif = true;
    else if (g.model == M_IAF_PSC_EXP || g.model == M_SPIKE_GEN || g.model == M_PARROT ||
             g.model == M_SPIKE_DET)
      has_other = true;
  }
  const bool fork = has_aeif && has_other;
  // Programmatic dependent launch where the batch is one chain of kernels on one stream
  // (no event edges between streams, no plastic-edge kernels, no per-kernel timing events).
  // (automatic: for one-step batches, where a step is two short launches and their launch
  // latency shows; longer batches measured slower with it)
  const bool pdl = launch_pdl > 0 || (launch_pdl < 0 && M == 1);
  set_launch_pdl(pdl && !fork && !plastic_ && !ev);
  if (ev) cuda_check(cudaEventRecord((*ev)[0], stream_), "event");
  if (plastic_) count_launch(launch_stdp_reset(stdp_, d_clk_, k0, stream_));
  // (delivery at emission: the update kernels deliver; there is no delivery launch)
  if (!push_)
    count_launch(launch_deliver(deliver_args(), deliver_blocks_req > 0 ? deliver_blocks_req : deliver_blocks_,
                                deliver_group, d_clk_, k0, M, stream_));
  if (ev) cuda_check(cudaEventRecord((*ev)[1], stream_), "event");
  cudaStream_t s2 = stream_;
  if (fork) {
    cuda_check(cudaEventRecord(ev_fork_, stream_), "fork");
    cuda_check(cudaStreamWaitEvent(stream2_, ev_fork_, 0), "fork");
    s2 = stream2_;
  }
  if (n_iaf_multi_ >= 2)
    count_launch(launch_iaf_multi(d_iaf_tab_, d_iaf_blk0_, n_iaf_multi_, iaf_multi_blocks_, so, push_ ? &po : nullptr,
                                  d_clk_, k0, M, s2));
  for (auto &g : groups_) {
    if (g.model == M_IAF_PSC_EXP && n_iaf_multi_ < 2)
      count_launch(launch_iaf(iaf_args(g), so, push_ ? &po : nullptr, d_clk_, k0, M, s2));
    else if (g.model == M_SPIKE_GEN) count_launch(launch_spike_gen(sg_args(g), so, d_clk_, k0, M, s2));
    else if (g.model == M_PARROT) count_launch(launch_parrot(parrot_args(g), so, d_clk_, k0, M, s2));
    else if (g.model == M_SPIKE_DET) count_launch(launch_spike_det(parrot_args(g), so, d_clk_, k0, M, s2));
  }
  for (auto &g : groups_)
    if (is_aeif(g.model)) count_launch(launch_aeif(g.model, aeif_args(g), so, d_clk_, k0, M, stream_));
  if (fork) {
    cuda_check(cudaEventRecord(ev_join_, stream2_), "join");
    cuda_check(cudaStreamWaitEvent(stream_, ev_join_, 0), "join");
  }
  // plastic edges (one step per batch): the step's arrivals, then its post-synaptic spikes
  if (plastic_) {
    if (d_rev_ring_)
      count_launch(launch_rev_arrivals(d_rev_ring_, d_rev_cnt_, rev_R_, rev_cap_, d_last_rev_, d_clk_, k0, stream_));
    count_launch(launch_stdp_forward(stdp_, d_clk_, k0, stream_));
    count_launch(launch_stdp_reverse(stdp_, d_clk_, k0, stream_));
  }
  if (ev) cuda_check(cudaEventRecord((*ev)[2], stream_), "event");
  set_launch_pdl(false);
}

// Argument table of the iaf groups for the single multi-group launch; rebuilt before
// each graph capture (the arguments hold record-buffer pointers that can change).
void Engine::prepare_multi() {
  std::vector<IafArgs> tab;
  std::vector<int> blk0, first{0};
  int nb = 0;
  for (auto &g : groups_) {
    if (g.model != M_IAF_PSC_EXP || g.n <= 0) continue;
    tab.push_back(iaf_args(g));
    blk0.push_back(nb);
    nb += (g.hi - g.lo + 255) / 256;
    first.push_back(first.back() + g.n);
  }
  n_iaf_multi_ = (int)tab.size();
  iaf_multi_blocks_ = nb;
  if (n_iaf_multi_ < 1) return;
  if (!d_iaf_tab_) {
    d_iaf_tab_ = dalloc<IafArgs>(tab.size());
    d_iaf_blk0_ = dalloc<int>(blk0.size());
    d_iaf_first_ = dalloc<int>(first.size());
    d_bar_ = dalloc<GridBarrier>(1);
  }
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  cuda_check(cudaMemcpy(d_iaf_tab_, tab.data(), tab.size() * sizeof(IafArgs), cudaMemcpyHostToDevice), "iaf table");
  cuda_check(cudaMemcpy(d_iaf_blk0_, blk0.data(), blk0.size() * sizeof(int), cudaMemcpyHostToDevice), "iaf table");
  cuda_check(cudaMemcpy(d_iaf_first_, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice),
             "iaf table");
}

// The persistent step loop serves networks whose only neurons are iaf_psc_exp groups
// (Poisson generators have no kernel of their own).
bool Engine::persistent_eligible() const {
  if (plastic_ || part_world_ > 1 || push_) return false;
  bool any = false;
  for (auto &g : groups_) {
    if (g.n <= 0 || g.model == M_POISS_GEN) continue;
    if (g.model != M_IAF_PSC_EXP) return false;
    any = true;
  }
  return any;
}

// Delivery at emission serves the same networks as the persistent loop: iaf_psc_exp groups
// only (their spikes have height 1 and their kernel is the only spike source), no plastic
// edges, one process.
bool Engine::push_eligible() const {
  if (plastic_ || part_world_ > 1) return false;
  bool any = false;
  for (auto &g : groups_) {
    if (g.n <= 0 || g.model == M_POISS_GEN) continue;
    if (g.model != M_IAF_PSC_EXP) return false;
    any = true;
  }
  return any;
}

// `steps` steps in one cooperative launch of the persistent loop, then the clock advance.
void Engine::run_persistent(int steps) {
  cuda_check(cudaMemsetAsync(d_bar_, 0, sizeof(GridBarrier), stream_), "barrier reset");
  const int r = launch_persistent_iaf(deliver_args(), deliver_group, d_iaf_tab_, d_iaf_first_, n_iaf_multi_,
                                      spike_out(), d_clk_, steps, batch_, d_bar_,
                                      deliver_blocks_req > 0 ? deliver_blocks_req : 0, barrier_extra, stream_);
  if (r < 0) throw NgpuError(std::string("cooperative launch of the persistent step loop failed: ") +
                             cudaGetErrorString(cudaGetLastError()));
  launch_clock_advance(d_clk_, steps, stream_);
  n_launch_ += 2;
}

void Engine::ensure_record_window(long long rows) {
  if (!rec_ncol_ || rows <= rec_rows_cap_) return;
  d_recbuf_ = dalloc<float>((size_t)rows * rec_ncol_);
  rec_rows_cap_ = (int)rows;
  invalidate_graphs();
}

void Engine::set_partition(int rank, int world) {
  if (calibrated_) throw NgpuError("the partition must be set before calibration");
  if (world < 1 || rank < 0 || rank >= world) throw NgpuError("partition rank out of range");
  part_rank_ = rank;
  part_world_ = world;
}

void Engine::set_exchange(void *send, void *recv, long long cap, int (*exchange)(void *), void *user) {
  if (cap < 1 || cap > (1LL << 30)) throw NgpuError("exchange capacity out of range");
  if (!send || !recv || !exchange) throw NgpuError("exchange buffers and function are required");
  if (((uintptr_t)send | (uintptr_t)recv) & 15) throw NgpuError("exchange buffers must be 16-byte aligned");
  xch_send_ = (int4 *)send;
  xch_recv_ = (int4 *)recv;
  xch_cap_ = (int)cap;
  xch_fn_ = exchange;
  xch_user_ = user;
  invalidate_graphs();
}

// Partitioned network: batch by batch (no graphs), each followed by the spike exchange:
// the batch's kernels, a wait for them, the caller's all-gather of the exchange buffers, the
// other processes' spikes into this process's ring, and the clock advance.  Every process
// runs the same batches, so the exchange calls pair up.
void Engine::run_batches_partitioned(long long n) {
  if (!xch_fn_) throw NgpuError("a partitioned network needs its exchange (NGPU_SetExchange) before simulating");
  const int M = batch_;
  long long window = n;
  const long long REC_WINDOW = 10000;
  if (rec_ncol_) {
    window = std::min<long long>(n, REC_WINDOW);
    ensure_record_window(window);
  }
  long long done = 0;
  while (done < n) {
    const long long w = std::min(window, n - done);
    for (long long left = w; left > 0;) {
      const int mb = (int)std::min<long long>(M, left);
      launch_batch(0, mb, nullptr);
      cuda_check(cudaStreamSynchronize(stream_), "batch");
      if (xch_fn_(xch_user_) != 0) throw NgpuError("the spike exchange failed");
      count_launch(launch_exchange_unpack(spike_out(), xch_recv_, xch_cap_, part_world_, part_rank_, stream_));
      count_launch(launch_clock_advance(d_clk_, mb, stream_));
      left -= mb;
    }
    if (rec_ncol_) drain_records(w);
    done += w;
  }
}

void Engine::run_steps(long long n) {
  if (part_world_ > 1) {
    run_batches_partitioned(n);
    return;
  }
  const int M = batch_;
  const int K = std::max(M, (std::max(1, graph_steps) / M) * M);   // steps per graph
  long long window = n;
  const long long REC_WINDOW = 10000;
  if (rec_ncol_) {
    window = std::min<long long>(n, REC_WINDOW);
    ensure_record_window(window);
  }
  const bool pers = persistent && persistent_eligible();
  if (pers) prepare_multi();
  long long done = 0;
  while (done < n) {
    const long long w = std::min(window, n - done);
    long long left = w;
    while (left > 0) {
      const int steps = (int)std::min<long long>(K, left);
      if (pers) {
        run_persistent(steps);
        left -= steps;
        continue;
      }
      auto itg = graphs_.find(steps);
      if (itg == graphs_.end()) {
        prepare_multi();
        cudaGraph_t graph;
        cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
        capturing_ = true;
        capture_count_ = 0;
        for (int k0 = 0; k0 < steps; k0 += M) launch_batch(k0, std::min(M, steps - k0), nullptr);
        count_launch(launch_clock_advance(d_clk_, steps, stream_));
        capturing_ = false;
        graph_nodes_[steps] = capture_count_;
        cuda_check(cudaStreamEndCapture(stream_, &graph), "capture");
        cudaGraphExec_t exec;
        cuda_check(cudaGraphInstantiate(&exec, graph, 0), "instantiate");
        cudaGraphDestroy(graph);
        itg = graphs_.emplace(steps, exec).first;
      }
      cuda_check(cudaGraphLaunch(itg->second, stream_), "graph launch");
      n_launch_ += graph_nodes_[steps];
      left -= steps;
    }
    if (rec_ncol_) drain_records(w);
    done += w;
  }
}

void Engine::drain_records(long long rows) {
  std::vector<float> buf((size_t)rows * rec_ncol_);
  cuda_check(cudaMemcpyAsync(buf.data(), d_recbuf_, buf.size() * sizeof(float), cudaMemcpyDeviceToHost,
                             stream_), "record copy");
  cuda_check(cudaStreamSynchronize(stream_), "record sync");
  // the next window starts where this one ended
  Clock c;
  cuda_check(cudaMemcpy(&c, d_clk_, sizeof(Clock), cudaMemcpyDeviceToHost), "clock");
  const long long it_first = c.rec_it0;
  c.rec_it0 = c.it0;
  cuda_check(cudaMemcpy(d_clk_, &c, sizeof(Clock), cudaMemcpyHostToDevice), "clock");
  for (long long r = 0; r < rows; r++) {
    const float *row = &buf[(size_t)r * rec_ncol_];
    // time of the step, as the reference writes it (float of the neural time)
    const float t = (float)(neur_t0_ + (double)dt * (double)(it_first + r + 1));
    size_t c0 = 0;
    for (auto &rs : records_) {
      std::vector<float> v;
      v.push_back(t);
      for (size_t c2 = 0; c2 < rs.var.size(); c2++) v.push_back(row[c0 + c2]);
      c0 += rs.var.size();
      if (rs.fp) {
        fprintf(rs.fp, "%f", v[0]);
        for (size_t j = 1; j < v.size(); j++) fprintf(rs.fp, "\t%f", v[j]);
        fprintf(rs.fp, "\n");
      }
      rs.data.push_back(std::move(v));
    }
  }
}

void Engine::drain_rec_spike_times() {
  if (!calibrated_) return;
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  for (auto &g : groups_) {
    if (g.max_rec <= 0 || !g.d_n_rec) continue;
    std::vector<int> nr(g.n);
    cuda_check(cudaMemcpy(nr.data(), g.d_n_rec, g.n * sizeof(int), cudaMemcpyDeviceToHost), "n_rec");
    int any = 0;
    for (int v : nr) any |= v;
    if (!any) continue;
    std::vector<float> t((size_t)g.n * g.max_rec);
    cuda_check(cudaMemcpy(t.data(), g.d_rec_times, t.size() * sizeof(float), cudaMemcpyDeviceToHost), "rec");
    for (int i = 0; i < g.n; i++)
      g.rec_times_host[i].insert(g.rec_times_host[i].end(), t.begin() + (size_t)i * g.max_rec,
                                 t.begin() + (size_t)i * g.max_rec + nr[i]);
    cuda_check(cudaMemset(g.d_n_rec, 0, g.n * sizeof(int)), "n_rec");
  }
}

void Engine::check_status() {
  unsigned st = 0;
  cuda_check(cudaMemcpy(&st, d_status_, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
  unsigned fresh = st & ~status_seen_;
  status_seen_ |= st;
  if (fresh && verbosity >= 1) {
    if (fresh & ST_RING_OVERFLOW) printf("Warning: spike ring slot overflow, spikes dropped\n");
    if (fresh & ST_RK5_TRIALS) printf("Warning: RK5 step hit its iteration cap\n");
    if (fresh & ST_NUMERIC) printf("Warning: V_m or w out of bounds, neuron state reset\n");
    if (fresh & ST_REC_TIMES_FULL) printf("Maximum number of recorded spike times exceeded\n");
  }
  if (st & ST_BARRIER_TIMEOUT) {
    // the loop stopped early: the state is not that of the requested time
    const unsigned keep = st & ~ST_BARRIER_TIMEOUT;
    cuda_check(cudaMemcpy(d_status_, &keep, sizeof(unsigned), cudaMemcpyHostToDevice), "status");
    status_seen_ &= ~ST_BARRIER_TIMEOUT;
    persistent = 0;
    throw NgpuError("a grid barrier of the persistent step loop timed out; the simulation state is invalid "
                    "(the engine falls back to per-batch launches)");
  }
}

void Engine::upload_dirty_params() {
  for (auto &g : groups_)
    if (g.dirty) {
      upload_params();
      return;
    }
}

void Engine::start_simulation() {
  if (!calibrated_) calibrate();
  if (in_sim_) {
    upload_dirty_params();
    return;
  }
  upload_params();
  if (first_sim_) {
    // initial record row (src/nestgpu.cu:384-389)
    for (auto &rs : records_) {
      std::vector<float> v{(float)neural_time_};
      for (size_t c = 0; c < rs.var.size(); c++) {
        if (rs.var[c] == "spike") {
          v.push_back(0.0f);
        } else {
          std::vector<float> x = get_values({rs.node[c]}, rs.var[c]);
          v.push_back(locate(rs.node[c], rs.var[c]) == K_PORT_VAR ? x[rs.port[c]] : x[0]);
        }
      }
      if (rs.fp) {
        fprintf(rs.fp, "%f", v[0]);
        for (size_t j = 1; j < v.size(); j++) fprintf(rs.fp, "\t%f", v[j]);
        fprintf(rs.fp, "\n");
      }
      rs.data.push_back(v);
    }
    first_sim_ = false;
  }
  if (verbosity >= 1) printf("Simulating ...\nNeural activity simulation time: %.3lf ms\n", (double)sim_time);
  neur_t0_ = neural_time_;
  it_ = 0;
  Nt_ = (long long)roundf(sim_time / dt);
  tidx_base_ = (long long)(int)std::round(neur_t0_ / (double)dt);
  Clock c;
  std::memset(&c, 0, sizeof(c));
  c.it0 = 0;
  c.tidx_base = tidx_base_;
  c.t0 = neur_t0_;
  c.rec_it0 = 0;
  cuda_check(cudaMemcpy(d_clk_, &c, sizeof(Clock), cudaMemcpyHostToDevice), "clock");
  in_sim_ = true;
}

void Engine::end_simulation() {
  if (!in_sim_) return;
  cuda_check(cudaStreamSynchronize(stream_), "end of simulation");
  drain_rec_spike_times();
  if (it_ > 0) neural_time_ = neur_t0_ + (double)dt * (double)it_;
  in_sim_ = false;
  check_status();
}

void Engine::simulation_step() {
  if (!in_sim_) start_simulation();
  // parameters set between steps apply from the next step, as the reference's setters
  // write to the device at once (src/base_neuron.cu:219-260)
  upload_dirty_params();
  // every step ends with its input fold, so state queries between steps see what the
  // reference shows
  run_steps(1);
  it_ += 1;
  cuda_check(cudaStreamSynchronize(stream_), "step");
  Clock c;
  cuda_check(cudaMemcpy(&c, d_clk_, sizeof(Clock), cudaMemcpyDeviceToHost), "clock");
  neural_time_ = neur_t0_ + (double)dt * (double)it_;
}

void Engine::simulate(float t) {
  sim_time = t;
  start_simulation();
  if (!ev_a_) {
    cuda_check(cudaEventCreate(&ev_a_), "event");
    cuda_check(cudaEventCreate(&ev_b_), "event");
  }
  auto t0 = std::chrono::steady_clock::now();
  cuda_check(cudaEventRecord(ev_a_, stream_), "event");
  run_steps(Nt_);
  it_ += Nt_;
  cuda_check(cudaEventRecord(ev_b_, stream_), "event");
  end_simulation();
  float ms = 0.0f;
  cuda_check(cudaEventElapsedTime(&ms, ev_a_, ev_b_), "event");
  last_sim_device_ms_ = ms;
  auto t1 = std::chrono::steady_clock::now();
  last_sim_seconds_ = std::chrono::duration<double>(t1 - t0).count();
  total_steps_ += Nt_;
  if (verbosity >= 1) printf("Simulation time: %g\n", last_sim_seconds_);
}

void Engine::delivery_shape(int *n_nodes_out, int *dmin, int *dspan, long long *n_edges) {
  if (!calibrated_) throw NgpuError("the delivery layout exists after calibration");
  if (n_nodes_out) *n_nodes_out = n_nodes();
  if (dmin) *dmin = dmin_;
  if (dspan) *dspan = dspan_;
  if (n_edges) *n_edges = (long long)n_edge_dev_;
}

void Engine::delivery_csr(long long *seg_off, int *target, unsigned char *port, float *weight) {
  if (!calibrated_) throw NgpuError("the delivery layout exists after calibration");
  const size_t nkey = (size_t)n_nodes() * dspan_;
  cuda_check(cudaStreamSynchronize(stream_), "sync");
  cuda_check(cudaMemcpy(seg_off, d_ev_off_, (nkey + 1) * sizeof(long long), cudaMemcpyDeviceToHost), "seg_off");
  std::vector<EdgeW> ew(n_edge_dev_);
  if (n_edge_dev_)
    cuda_check(cudaMemcpy(ew.data(), d_edge_, n_edge_dev_ * sizeof(EdgeW), cudaMemcpyDeviceToHost), "edges");
  // accumulator index -> (target node, receptor port): groups own contiguous ranges
  std::vector<const Group *> by_off;
  for (auto &g : groups_)
    if (g.nport > 0) by_off.push_back(&g);
  std::sort(by_off.begin(), by_off.end(), [](const Group *a, const Group *b) { return a->acc_off < b->acc_off; });
  for (size_t e = 0; e < n_edge_dev_; e++) {
    const size_t a = ew[e].acc;
    size_t lo = 0, hi = by_off.size();
    while (hi - lo > 1) {
      const size_t mid = (lo + hi) / 2;
      if (by_off[mid]->acc_off <= a) lo = mid; else hi = mid;
    }
    const Group &g = *by_off[lo];
    const size_t r = a - g.acc_off;
    if (target) target[e] = g.i0 + (int)(r % g.n);
    if (port) port[e] = (unsigned char)(r / g.n);
    if (weight) weight[e] = ew[e].w;
  }
}

std::vector<double> Engine::profile_steps(int n) {
  if (in_sim_) throw NgpuError("profile_steps cannot run inside a simulation");
  sim_time = (float)n * dt;
  start_simulation();
  ensure_record_window(n);
  prepare_multi();
  std::vector<cudaEvent_t> ev(3);
  for (auto &e : ev) cuda_check(cudaEventCreate(&e), "event");
  std::vector<double> acc(3, 0.0);
  const int M = batch_;
  int done = 0;
  while (done < n) {
    const int mb = std::min(M, n - done);
    launch_batch(0, mb, &ev);
    if (part_world_ > 1) {
      // partitioned network: the batch's exchange, as in run_batches_partitioned
      cuda_check(cudaStreamSynchronize(stream_), "batch");
      if (!xch_fn_ || xch_fn_(xch_user_) != 0) throw NgpuError("the spike exchange failed");
      count_launch(launch_exchange_unpack(spike_out(), xch_recv_, xch_cap_, part_world_, part_rank_, stream_));
    }
    count_launch(launch_clock_advance(d_clk_, mb, stream_));
    cuda_check(cudaEventSynchronize(ev[2]), "event");
    float ms_del = 0.0f, ms_upd = 0.0f;
    cuda_check(cudaEventElapsedTime(&ms_del, ev[0], ev[1]), "event");
    cuda_check(cudaEventElapsedTime(&ms_upd, ev[1], ev[2]), "event");
    acc[0] += ms_upd;
    acc[2] += ms_del;
    done += mb;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  if (rec_ncol_) drain_records(n);
  it_ += n;
  end_simulation();
  total_steps_ += n;
  for (auto &a : acc) a /= std::max(1, n);
  return acc;
}

EngineStats Engine::stats() {
  EngineStats s;
  if (calibrated_) {
    unsigned long long c[4];
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    cuda_check(cudaMemcpy(c, d_counters_, sizeof(c), cudaMemcpyDeviceToHost), "counters");
    s.n_derivs = c[0];
    s.n_events = c[1];
    s.n_spikes = c[2];
    cuda_check(cudaMemcpy(&s.status, d_status_, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
  }
  s.sim_seconds = last_sim_seconds_;
  s.sim_device_ms = last_sim_device_ms_;
  s.steps = total_steps_;
  return s;
}

// ---------------------------------------------------------------------------
// Autotuner of the launch mappings
// ---------------------------------------------------------------------------
int Engine::autotune(int steps, std::vector<std::pair<std::string, double>> *log) {
  if (steps < 1) throw NgpuError("autotune needs at least one step per trial");
  if (in_sim_) throw NgpuError("autotune cannot run inside a simulation");
  if (!calibrated_) calibrate();
  const int verb = verbosity;
  verbosity = 0;
  const int base = std::max(148, deliver_blocks_);
  // A knob sets one or more variables together: the delivery lane group and grid interact
  // (a coordinate descent over them one at a time settles in local optima), so their
  // combinations are one knob.
  struct Knob {
    const char *name;
    std::vector<int *> vars;
    std::vector<std::vector<int>> cand;
  };
  auto single = [](const char *name, int *var, std::vector<int> vals) {
    Knob k{name, {var}, {}};
    for (int v : vals) k.cand.push_back({v});
    return k;
  };
  Knob deliver{"deliver_group,deliver_blocks", {&deliver_group, &deliver_blocks_req}, {}};
  std::vector<int> blocks{148, 296, 592, 1184, 2368};
  if (std::find(blocks.begin(), blocks.end(), base) == blocks.end()) blocks.push_back(base);
  for (int g : {8, 16, 32})
    for (int b : blocks) deliver.cand.push_back({g, b});
  std::vector<Knob> knobs = {
      single("update_threads", &update_threads, {64, 128, 256}),
      single("update_occupancy", &update_occupancy, {0, 1, 2}),
      single("update_trial_iter", &update_trial_iter, {0, 1}),
      single("deliver_aggregate", &deliver_aggregate, {0, 1}),
      single("deliver_prefetch", &deliver_prefetch, {0, 1}),
      deliver,
      single("rk5_budget", &rk5_budget, {0, 1, 2, 4, 8}),
      single("programmatic_launch", &launch_pdl, {0, 1}),
  };
  if (persistent_eligible()) knobs.insert(knobs.begin(), single("persistent", &persistent, {0, 1}));
  if (deliver_blocks_req <= 0) deliver_blocks_req = base;
  const float t = (float)steps * dt;
  auto trial = [&]() {
    invalidate_graphs();
    simulate(t);   // captures the graphs
    simulate(t);
    return last_sim_device_ms_;
  };
  int n_trials = 0;
  try {
    // A network started from rest goes through a transient in which its activity, and so
    // the cost of a step, changes from one trial to the next: run through it first.  Then
    // each knob's candidates are timed twice, in forward and in reverse order (a slow drift
    // of the activity then favours none of them), and the better time of each counts.
    simulate(4.0f * t);
    for (int pass = 0; pass < 2; pass++) {
      for (auto &k : knobs) {
        auto set = [&](const std::vector<int> &v) {
          for (size_t j = 0; j < k.vars.size(); j++) *k.vars[j] = v[j];
        };
        std::vector<std::vector<int>> cand;
        std::vector<int> cur;
        for (int *p : k.vars) cur.push_back(*p);
        cand.push_back(cur);
        for (auto &c : k.cand)
          if (c != cur) cand.push_back(c);
        std::vector<double> best_ms(cand.size(), 1e300);
        for (int rep = 0; rep < 2; rep++) {
          for (size_t u = 0; u < cand.size(); u++) {
            const size_t ci = rep == 0 ? u : cand.size() - 1 - u;
            set(cand[ci]);
            const double ms = trial();
            n_trials++;
            if (log) {
              std::string s = std::string(k.name) + "=";
              for (size_t j = 0; j < cand[ci].size(); j++) s += (j ? "," : "") + std::to_string(cand[ci][j]);
              log->push_back({s, ms});
            }
            best_ms[ci] = std::min(best_ms[ci], ms);
          }
        }
        size_t bi = 0;
        for (size_t ci = 1; ci < cand.size(); ci++)
          if (best_ms[ci] < best_ms[bi]) bi = ci;
        set(cand[bi]);
      }
    }
  } catch (...) {
    verbosity = verb;
    throw;
  }
  verbosity = verb;
  invalidate_graphs();
  return n_trials;
}

// ---------------------------------------------------------------------------
// Learned RK5 step-size proposal: logging, training, model
// ---------------------------------------------------------------------------
void Engine::set_learn_mode(int mode) {
  if (stream_) cuda_check(cudaStreamSynchronize(stream_), "sync");
  if (mode != learn_mode_) invalidate_graphs();
  learn_mode_ = mode;
}

void Engine::rk5_log_start(long long cap) {
  if (cap <= 0) throw NgpuError("RK5 log capacity must be positive");
  if (stream_) cuda_check(cudaStreamSynchronize(stream_), "sync");
  if (cap != log_cap_) {
    if (d_log_) cudaFree(d_log_);
    d_log_ = nullptr;
    log_cap_ = 0;
    cuda_check(cudaMalloc(&d_log_, (size_t)cap * LOG_W * sizeof(float)), "RK5 log buffer");
    log_cap_ = cap;
  }
  if (!d_log_cursor_) cuda_check(cudaMalloc(&d_log_cursor_, sizeof(unsigned long long)), "RK5 log cursor");
  cuda_check(cudaMemset(d_log_cursor_, 0, sizeof(unsigned long long)), "RK5 log cursor");
  invalidate_graphs();   // the log buffer is baked into captured kernel arguments
  set_learn_mode(LM_LOG);
}

void Engine::rk5_log_stop() {
  if (learn_mode_ == LM_LOG) set_learn_mode(LM_PLAIN);
}

long long Engine::rk5_log_count(long long *offered) {
  unsigned long long c = 0;
  if (d_log_cursor_) {
    if (stream_) cuda_check(cudaStreamSynchronize(stream_), "sync");
    cuda_check(cudaMemcpy(&c, d_log_cursor_, sizeof(c), cudaMemcpyDeviceToHost), "RK5 log cursor");
  }
  if (offered) *offered = (long long)c;
  return std::min<long long>((long long)c, log_cap_);
}

void Engine::rk5_log_get(float *out, long long first, long long n) {
  const long long have = rk5_log_count(nullptr);
  if (first < 0 || n < 0 || first + n > have) throw NgpuError("RK5 log range out of bounds");
  if (n == 0) return;
  cuda_check(cudaMemcpy(out, d_log_ + (size_t)first * LOG_W, (size_t)n * LOG_W * sizeof(float),
                        cudaMemcpyDeviceToHost), "RK5 log download");
}

TrainResult Engine::step_model_train(const TrainConfig &cfg) {
  const long long n = rk5_log_count(nullptr);
  if (n <= 0) throw NgpuError("no RK5 steps logged: call the RK5 log before training");
  std::vector<float> p(SM_NPAR);
  TrainResult r = train_step_model(d_log_, n, cfg, p.data());
  step_model_set(p.data());
  return r;
}

void Engine::step_model_set(const float *p) {
  for (int j = 0; j < SM_NPAR; j++)
    if (!(std::fabs(p[j]) < 3.0e38f)) throw NgpuError("step model parameter " + std::to_string(j) + " is not finite");
  if (!(p[SM_SAFETY] > 0.0f)) throw NgpuError("step model safety factor must be positive");
  if (!(p[SM_FLOOR] >= 0.0f)) throw NgpuError("step model floor must be >= 0");
  model_.assign(p, p + SM_NPAR);
  if (stream_) cuda_check(cudaStreamSynchronize(stream_), "sync");
  if (!d_model_) cuda_check(cudaMalloc(&d_model_, SM_NPAR * sizeof(float)), "step model");
  cuda_check(cudaMemcpy(d_model_, model_.data(), SM_NPAR * sizeof(float), cudaMemcpyHostToDevice), "step model");
  has_model_ = true;
  invalidate_graphs();
}

void Engine::step_model_get(float *p) const {
  if (!has_model_) throw NgpuError("no step model has been trained or set");
  std::copy(model_.begin(), model_.end(), p);
}

void Engine::step_bound_mode(bool on) { set_learn_mode(on ? LM_BOUND : LM_PLAIN); }

void Engine::step_model_enable(bool on) {
  if (on && !has_model_) throw NgpuError("no step model has been trained or set");
  set_learn_mode(on ? LM_PROPOSE : LM_PLAIN);
}

}  // namespace ngpu
