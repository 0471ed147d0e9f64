// Device-side construction of the recurrent CSR (edges sorted by (source, delay)).
//
// Edges come from two places: the host connection store (rule-based Connect
// calls, kept for GetConnections) and generated blocks (fixed in-degree with
// per-target random sources and uniform delays on the time grid, drawn on the
// GPU from Philox4x32-10 so that 1e9-edge networks never touch host memory).
// Counting sort on the device: per-key counters, an exclusive scan into the
// segment offsets, host edges first in each segment (insertion order), then the
// generated edges through atomic cursors.  The order inside a segment does not
// change results: the input accumulator sums in FP64 and is read only after the
// delivery kernel has finished.
#include <cub/device/device_scan.cuh>

#include <stdexcept>
#include <string>
#include <vector>

#include "ngpu_math.cuh"
#include "ngpu_types.h"

namespace ngpu {


// Edge e = t*k + kk of a block: in-edge kk of the block's target t (0-based inside the
// block).  One Philox4x32-10 call keyed by the block's seed with counter (t, kk, 0,
// 0x9E3779B9): source = src0 + floor(x * nsrc / 2^32), delay step = dlo +
// floor(y * (dhi - dlo + 1) / 2^32).  Everything is relative to the block, so a block
// draws the same edges wherever its nodes sit in the network; blocks that should differ
// need different seeds.
__device__ __forceinline__ void gen_edge(const GenBlockDev &b, long long e, int &src, int &d, int &tgt) {
  const int t = (int)(e / b.k);
  const int kk = (int)(e - (long long)t * b.k);
  U4 c = {(uint32_t)t, (uint32_t)kk, 0u, 0x9E3779B9u};
  U4 r = philox(c, (uint32_t)b.seed, (uint32_t)(b.seed >> 32));
  src = b.src0 + (int)(((unsigned long long)r.x * (unsigned)b.nsrc) >> 32);
  d = b.dlo + (int)(((unsigned long long)r.y * (unsigned)(b.dhi - b.dlo + 1)) >> 32);
  tgt = t;
}

__global__ void gen_count_kernel(GenBlockDev b, int dmin, int dspan, unsigned long long *cnt) {
  const long long total = (long long)b.t_end * b.k;
  for (long long e = (long long)b.t_begin * b.k + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int s, d, t;
    gen_edge(b, e, s, d, t);
    atomicAdd(&cnt[(size_t)s * dspan + (d - dmin)], 1ULL);
  }
}

__global__ void gen_fill_kernel(GenBlockDev b, int dmin, int dspan, unsigned long long *cursor,
                                EdgeW *edge) {
  const long long total = (long long)b.t_end * b.k;
  for (long long e = (long long)b.t_begin * b.k + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int s, d, t;
    gen_edge(b, e, s, d, t);
    unsigned long long pos = atomicAdd(&cursor[(size_t)s * dspan + (d - dmin)], 1ULL);
    EdgeW x;
    x.acc = (uint32_t)(b.acc_base + (unsigned long long)(b.tgt_i0_rel + t));
    x.w = b.w;
    edge[pos] = x;
  }
}

// Edge e of a rule block (see RuleBlockDev): source and target nodes, weight, delay [ms].
__device__ __forceinline__ void rule_edge(const RuleBlockDev &b, long long e, int &src, int &tgt, float &w,
                                          float &d) {
  int is, it;
  if (b.rule == 2) {
    is = (int)(b.rnd[2 * e] % (unsigned)b.ns);
    it = (int)(b.rnd[2 * e + 1] % (unsigned)b.nt);
  } else {
    const long long kk = e / b.degree;
    const int i = (int)(e - kk * b.degree);
    if (b.rule == 3) {
      is = b.pick[i];
      it = (int)kk;
    } else {
      is = (int)kk;
      it = b.pick[i];
    }
  }
  src = b.src_arr ? b.src_arr[is] : b.src0 + is;
  tgt = b.tgt_arr ? b.tgt_arr[it] : b.tgt0 + it;
  w = b.warr ? b.warr[e] : b.w;
  d = b.darr ? b.darr[e] : b.d_ms;
}

// Delay step of a delay in ms: round(d / dt) - 1 (src/connect.cu:49), float arithmetic.
__device__ __forceinline__ int delay_step(float d, float dt) { return (int)roundf(__fdiv_rn(d, dt)) - 1; }

// node_acc0[t] == 0xffffffff marks a target simulated by another process (skipped)
__global__ void rule_count_kernel(RuleBlockDev b, int dmin, int dspan, unsigned long long *cnt,
                                  const unsigned *node_acc0) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < b.n_edges;
       e += (long long)gridDim.x * blockDim.x) {
    int s, t;
    float w, d;
    rule_edge(b, e, s, t, w, d);
    if (node_acc0[t] == 0xffffffffu) continue;
    atomicAdd(&cnt[(size_t)s * dspan + (delay_step(d, b.dt) - dmin)], 1ULL);
  }
}

__global__ void rule_fill_kernel(RuleBlockDev b, int dmin, int dspan, unsigned long long *cursor, EdgeW *edge,
                                 const unsigned *node_acc0, const int *node_gn) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < b.n_edges;
       e += (long long)gridDim.x * blockDim.x) {
    int s, t;
    float w, d;
    rule_edge(b, e, s, t, w, d);
    if (node_acc0[t] == 0xffffffffu) continue;
    const unsigned long long pos = atomicAdd(&cursor[(size_t)s * dspan + (delay_step(d, b.dt) - dmin)], 1ULL);
    EdgeW x;
    x.acc = node_acc0[t] + (unsigned)b.port * (unsigned)node_gn[t];
    x.w = w;
    edge[pos] = x;
  }
}

// Partitioned network: mark every source with a recurrent edge anywhere (all targets of the
// generated and rule blocks, not only those simulated here).
__global__ void gen_mark_kernel(GenBlockDev b, unsigned char *flag) {
  const long long total = (long long)b.ntgt * b.k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int s, d, t;
    gen_edge(b, e, s, d, t);
    flag[s] = 1;
  }
}

__global__ void rule_mark_kernel(RuleBlockDev b, unsigned char *flag) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < b.n_edges;
       e += (long long)gridDim.x * blockDim.x) {
    int s, t;
    float w, d;
    rule_edge(b, e, s, t, w, d);
    flag[s] = 1;
  }
}

void mark_sources_device(const std::vector<GenBlockDev> &blocks, const std::vector<RuleBlockDev> &rblocks,
                         unsigned char *d_flag, cudaStream_t st) {
  for (const auto &b : blocks) gen_mark_kernel<<<148 * 8, 256, 0, st>>>(b, d_flag);
  for (const auto &b : rblocks) rule_mark_kernel<<<148 * 8, 256, 0, st>>>(b, d_flag);
}

__global__ void host_edge_scatter_kernel(size_t n, const long long *key, const int *rank,
                                         const EdgeW *ew, const unsigned long long *off, EdgeW *edge) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    edge[off[key[i]] + rank[i]] = ew[i];
}

__global__ void cursor_init_kernel(size_t nkey, const unsigned long long *off, const int *cnt_host,
                                   unsigned long long *cursor) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nkey; i += (size_t)gridDim.x * blockDim.x)
    cursor[i] = off[i] + (cnt_host ? (unsigned long long)cnt_host[i] : 0ULL);
}

__global__ void has_out_kernel(int n_nodes, int dspan, const unsigned long long *off, unsigned char *has_out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_nodes; s += gridDim.x * blockDim.x)
    has_out[s] = off[(size_t)(s + 1) * dspan] > off[(size_t)s * dspan] ? 1 : 0;
}

static void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// Build the CSR.  cnt_host: per-key counts of host edges (or empty); host edges given as
// (key, rank in segment, EdgeW).  Returns device offsets (nkey+1, unsigned 64-bit) and edges.
void build_csr_device(int n_nodes, int dmin, int dspan, const std::vector<int> &cnt_host,
                      const std::vector<long long> &h_key, const std::vector<int> &h_rank,
                      const std::vector<EdgeW> &h_ew, const std::vector<GenBlockDev> &blocks,
                      const std::vector<RuleBlockDev> &rblocks, const unsigned *d_node_acc0,
                      const int *d_node_gn, unsigned long long **d_off_out, EdgeW **d_edge_out,
                      size_t *n_edge_out, unsigned char *d_has_out, cudaStream_t st) {
  const size_t nkey = (size_t)n_nodes * dspan;
  unsigned long long *d_cnt = nullptr, *d_off = nullptr, *d_cursor = nullptr;
  int *d_cnt_host = nullptr;
  ck(cudaMalloc(&d_cnt, (nkey + 1) * sizeof(unsigned long long)), "cudaMalloc");
  ck(cudaMalloc(&d_off, (nkey + 1) * sizeof(unsigned long long)), "cudaMalloc");
  ck(cudaMemsetAsync(d_cnt, 0, (nkey + 1) * sizeof(unsigned long long), st), "memset");
  if (!cnt_host.empty()) {
    ck(cudaMalloc(&d_cnt_host, nkey * sizeof(int)), "cudaMalloc");
    ck(cudaMemcpyAsync(d_cnt_host, cnt_host.data(), nkey * sizeof(int), cudaMemcpyHostToDevice, st), "copy");
    std::vector<unsigned long long> c64(cnt_host.begin(), cnt_host.end());
    ck(cudaMemcpyAsync(d_cnt, c64.data(), nkey * sizeof(unsigned long long), cudaMemcpyHostToDevice, st), "copy");
    ck(cudaStreamSynchronize(st), "sync");
  }
  const int gb = 148 * 8, tb = 256;
  for (const auto &b : blocks) gen_count_kernel<<<gb, tb, 0, st>>>(b, dmin, dspan, d_cnt);
  for (const auto &b : rblocks) rule_count_kernel<<<gb, tb, 0, st>>>(b, dmin, dspan, d_cnt, d_node_acc0);
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_cnt, d_off, nkey + 1, st);
  void *d_tmp = nullptr;
  ck(cudaMalloc(&d_tmp, tmp_bytes), "cudaMalloc");
  cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_cnt, d_off, nkey + 1, st);
  unsigned long long total = 0;
  ck(cudaMemcpyAsync(&total, d_off + nkey, sizeof(total), cudaMemcpyDeviceToHost, st), "copy");
  ck(cudaStreamSynchronize(st), "sync");
  EdgeW *d_edge = nullptr;
  ck(cudaMalloc(&d_edge, std::max<unsigned long long>(total, 1) * sizeof(EdgeW)), "cudaMalloc (edges)");
  if (!h_ew.empty()) {
    long long *d_key = nullptr;
    int *d_rank = nullptr;
    EdgeW *d_hew = nullptr;
    size_t n = h_ew.size();
    ck(cudaMalloc(&d_key, n * sizeof(long long)), "cudaMalloc");
    ck(cudaMalloc(&d_rank, n * sizeof(int)), "cudaMalloc");
    ck(cudaMalloc(&d_hew, n * sizeof(EdgeW)), "cudaMalloc");
    ck(cudaMemcpyAsync(d_key, h_key.data(), n * sizeof(long long), cudaMemcpyHostToDevice, st), "copy");
    ck(cudaMemcpyAsync(d_rank, h_rank.data(), n * sizeof(int), cudaMemcpyHostToDevice, st), "copy");
    ck(cudaMemcpyAsync(d_hew, h_ew.data(), n * sizeof(EdgeW), cudaMemcpyHostToDevice, st), "copy");
    host_edge_scatter_kernel<<<gb, tb, 0, st>>>(n, d_key, d_rank, d_hew, d_off, d_edge);
    ck(cudaStreamSynchronize(st), "scatter");
    cudaFree(d_key);
    cudaFree(d_rank);
    cudaFree(d_hew);
  }
  if (!blocks.empty() || !rblocks.empty()) {
    ck(cudaMalloc(&d_cursor, nkey * sizeof(unsigned long long)), "cudaMalloc");
    cursor_init_kernel<<<gb, tb, 0, st>>>(nkey, d_off, d_cnt_host, d_cursor);
    for (const auto &b : blocks) gen_fill_kernel<<<gb, tb, 0, st>>>(b, dmin, dspan, d_cursor, d_edge);
    for (const auto &b : rblocks)
      rule_fill_kernel<<<gb, tb, 0, st>>>(b, dmin, dspan, d_cursor, d_edge, d_node_acc0, d_node_gn);
  }
  has_out_kernel<<<gb, tb, 0, st>>>(n_nodes, dspan, d_off, d_has_out);
  ck(cudaStreamSynchronize(st), "build");
  ck(cudaGetLastError(), "build kernels");
  cudaFree(d_tmp);
  cudaFree(d_cnt);
  if (d_cursor) cudaFree(d_cursor);
  if (d_cnt_host) cudaFree(d_cnt_host);
  *d_off_out = d_off;
  *d_edge_out = d_edge;
  *n_edge_out = (size_t)total;
}

// ---------------------------------------------------------------------------
// Standalone packing of a device edge list into the delivery layout.
// ---------------------------------------------------------------------------
__global__ void list_count_kernel(size_t n, const int *src, const int *dly, int n_nodes, int dspan,
                                  unsigned long long *cnt, unsigned *bad) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int s = src[e], d = dly[e];
    if (s < 0 || s >= n_nodes || d < 0 || d >= dspan) {
      atomicOr(bad, 1u);
      continue;
    }
    atomicAdd(&cnt[(size_t)s * dspan + d], 1ULL);
  }
}

__global__ void list_fill_kernel(size_t n, const int *src, const int *dly, const unsigned *target,
                                 const float *weight, int n_nodes, int dspan, unsigned long long *cursor,
                                 EdgeW *edge) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int s = src[e], d = dly[e];
    if (s < 0 || s >= n_nodes || d < 0 || d >= dspan) continue;
    const unsigned long long pos = atomicAdd(&cursor[(size_t)s * dspan + d], 1ULL);
    EdgeW x;
    x.acc = target[e];
    x.w = weight[e];
    edge[pos] = x;
  }
}

// Counting sort with scratch from cudaMalloc: counters, cursors, scan workspace.
void pack_delivery_csr(const int *src, const int *dly, const unsigned *target, const float *weight,
                       size_t n, int n_nodes, int dspan, unsigned long long *seg_off, EdgeW *edge,
                       cudaStream_t st) {
  const size_t nkey = (size_t)n_nodes * dspan;
  unsigned long long *d_cnt = nullptr;
  unsigned *d_bad = nullptr;
  void *d_tmp = nullptr;
  size_t tmp_bytes = 0;
  ck(cudaMalloc(&d_cnt, (nkey + 1) * sizeof(unsigned long long) + 256), "cudaMalloc");
  d_bad = (unsigned *)(d_cnt + nkey + 1);
  ck(cudaMemsetAsync(d_cnt, 0, (nkey + 1) * sizeof(unsigned long long) + sizeof(unsigned), st), "memset");
  const int gb = 148 * 8, tb = 256;
  list_count_kernel<<<gb, tb, 0, st>>>(n, src, dly, n_nodes, dspan, d_cnt, d_bad);
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_cnt, seg_off, nkey + 1, st);
  ck(cudaMalloc(&d_tmp, tmp_bytes), "cudaMalloc");
  cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_cnt, seg_off, nkey + 1, st);
  // the counters become the fill cursors
  ck(cudaMemcpyAsync(d_cnt, seg_off, nkey * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st), "copy");
  list_fill_kernel<<<gb, tb, 0, st>>>(n, src, dly, target, weight, n_nodes, dspan, d_cnt, edge);
  unsigned bad = 0;
  ck(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "copy");
  ck(cudaStreamSynchronize(st), "pack");
  ck(cudaGetLastError(), "pack kernels");
  cudaFree(d_tmp);
  cudaFree(d_cnt);
  if (bad) throw std::runtime_error("edge list holds a source or delay index out of range");
}

}  // namespace ngpu
