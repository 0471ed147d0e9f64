// Learned RK5 step-size proposal: the logging / proposing variants of the aeif
// kernels and the MLP kernels that train the proposal network on the GPU.
//
// Training (per iteration, minibatch of B sampled tuples):
//   mlp_grad_kernel    one 128-sample tile per block: each thread runs the forward
//                      and backward pass of one sample with the BF16 weights,
//                      keeping inputs, activations and back-propagated errors in
//                      shared memory; the block then forms its weight gradients as
//                      sums over the tile's samples (dW = sum_s delta_s a_s^T), FP32,
//                      in a fixed order, and writes one partial gradient row;
//   reduce_kernel      sums the partial rows in block order (deterministic);
//   adam_kernel        Adam update of the FP32 master weights; the weights the
//                      network runs with are their BF16 roundings.
// The tuples are first filtered (only steps where the plain h would not reach the
// end of the time step are ones the network is asked about) and turned into
// (features, target) pairs, and the feature / target moments are reduced on the GPU.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "ngpu_aeif.cuh"
#include "ngpu_engine.h"

namespace ngpu {

// ---------------------------------------------------------------------------
// aeif kernels with logging or proposal (fixed port counts 1..4)
// ---------------------------------------------------------------------------
template <int MODEL, int LM>
static int launch_learn_m(const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                          cudaStream_t st) {
  switch (A.nport) {
  case 1: return launch_aeif_p<MODEL, 1, true, LM>(A, so, clk, k0, M, st);
  case 2: return launch_aeif_p<MODEL, 2, true, LM>(A, so, clk, k0, M, st);
  case 3: return launch_aeif_p<MODEL, 3, true, LM>(A, so, clk, k0, M, st);
  case 4: return launch_aeif_p<MODEL, 4, true, LM>(A, so, clk, k0, M, st);
  }
  throw NgpuError("the learned step-size path supports 1 to 4 receptor ports");
}

template <int LM>
static int launch_learn_l(int model, const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                          cudaStream_t st) {
  switch (model) {
  case M_AEIF_COND_BETA: return launch_learn_m<M_AEIF_COND_BETA, LM>(A, so, clk, k0, M, st);
  case M_AEIF_COND_ALPHA: return launch_learn_m<M_AEIF_COND_ALPHA, LM>(A, so, clk, k0, M, st);
  case M_AEIF_PSC_EXP: return launch_learn_m<M_AEIF_PSC_EXP, LM>(A, so, clk, k0, M, st);
  case M_AEIF_PSC_ALPHA: return launch_learn_m<M_AEIF_PSC_ALPHA, LM>(A, so, clk, k0, M, st);
  }
  return 0;
}

int launch_aeif_learn(int model, const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                      cudaStream_t st) {
  if (A.learn.mode == LM_LOG) return launch_learn_l<LM_LOG>(model, A, so, clk, k0, M, st);
  if (A.learn.mode == LM_BOUND) return launch_learn_l<LM_BOUND>(model, A, so, clk, k0, M, st);
  return launch_learn_l<LM_PROPOSE>(model, A, so, clk, k0, M, st);
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static void cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw NgpuError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// Round to the nearest BF16 value, ties to even; returned as a float.
__host__ __device__ inline float bf16_round_bits(uint32_t u, bool &special) {
  special = (u & 0x7f800000u) == 0x7f800000u;
  if (!special) u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float f;
#ifdef __CUDA_ARCH__
  f = __uint_as_float(u);
#else
  memcpy(&f, &u, 4);
#endif
  return f;
}
__device__ __forceinline__ float bf16_round(float v) {
  bool sp;
  return bf16_round_bits(__float_as_uint(v), sp);
}
static float bf16_round_host(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  bool sp;
  return bf16_round_bits(u, sp);
}

static inline bool is_weight(int j) {   // j: index into the flat parameter vector
  return (j >= SM_W1 && j < SM_B1) || (j >= SM_W2 && j < SM_B2) || (j >= SM_W3 && j < SM_B3);
}

// ---------------------------------------------------------------------------
// tuple filtering and moments
// ---------------------------------------------------------------------------
// Target of a logged step and whether the network would be consulted on it.
__device__ __forceinline__ bool tuple_target(const float *t, float &target) {
  const float lerr = log_m(fmaxf(t[SM_NF + 1], 1.889568e-4f));
  target = __fmaf_rn(-0.2f, lerr, log_m(t[SM_NF]));
  bool ok = t[8] < t[9] && target == target && fabsf(target) < 1.0e30f;
#pragma unroll
  for (int k = 0; k < SM_NF; k++) ok = ok && (fabsf(t[k]) < 1.0e30f);
  return ok;
}

__global__ void tuple_flag_kernel(const float *tuples, long long n, int *flag) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    float tg;
    flag[s] = tuple_target(tuples + s * LOG_W, tg) ? 1 : 0;
  }
}

// Usable tuple s goes to row pos[s] (exclusive scan of the flags): stable order.
__global__ void tuple_scatter_kernel(const float *tuples, long long n, const int *flag, const int *pos, float *feat,
                                     float *target) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    if (!flag[s]) continue;
    const float *t = tuples + s * LOG_W;
    const long long r = pos[s];
    float tg;
    tuple_target(t, tg);
    target[r] = tg;
#pragma unroll
    for (int k = 0; k < SM_NF; k++) feat[r * SM_NF + k] = t[k];
  }
}

// Per-block sums of x and x^2 for the 10 features and the target, in FP64.
constexpr int MOM_W = 2 * (SM_NF + 1);
__global__ void moments_kernel(const float *feat, const float *target, long long n, double *partial) {
  double acc[MOM_W];
#pragma unroll
  for (int k = 0; k < MOM_W; k++) acc[k] = 0.0;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k <= SM_NF; k++) {
      const double v = (k < SM_NF) ? (double)feat[s * SM_NF + k] : (double)target[s];
      acc[2 * k] += v;
      acc[2 * k + 1] = __fma_rn(v, v, acc[2 * k + 1]);
    }
  }
  __shared__ double red[MOM_W][256];
#pragma unroll
  for (int k = 0; k < MOM_W; k++) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < MOM_W; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < MOM_W) partial[blockIdx.x * MOM_W + threadIdx.x] = red[threadIdx.x][0];
}

// ---------------------------------------------------------------------------
// forward (inference) over a feature array
// ---------------------------------------------------------------------------
__global__ void mlp_forward_kernel(const float *model, const float *feat, int n, float *out) {
  __shared__ float M[SM_NPAR];
  for (int j = threadIdx.x; j < SM_NPAR; j += blockDim.x) M[j] = model[j];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    float f[SM_NF];
#pragma unroll
    for (int k = 0; k < SM_NF; k++) f[k] = feat[(size_t)s * SM_NF + k];
    out[s] = mlp_out(M, f);
  }
}

// ---------------------------------------------------------------------------
// gradient of the mean squared error over one tile of samples per block
// ---------------------------------------------------------------------------
constexpr int GT = 128;                  // samples per tile = threads per block
constexpr int RS = SM_NH + 1;            // padded row stride of the activation tiles
constexpr int PART_W = SM_NTRAIN + 1;    // partial row: gradients, then the loss sum
constexpr size_t GRAD_SMEM = sizeof(float) * ((size_t)SM_NPAR + GT * SM_NF + 4 * GT * RS + GT);

__device__ __forceinline__ uint32_t sample_index(uint64_t seed, long long iter, int s, uint32_t n) {
  U4 c{(uint32_t)s, (uint32_t)iter, (uint32_t)((unsigned long long)iter >> 32), 0x51ed2701u};
  U4 r = philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return (uint32_t)(((unsigned long long)r.x * n) >> 32);
}

// Samples: tile blockIdx.x covers batch positions [GT*blockIdx.x, GT*blockIdx.x+GT) of B;
// position s uses sample sample_index(seed, iter, s) if sampled, else sample s.
__global__ void __launch_bounds__(GT) mlp_grad_kernel(const float *model, const float *feat, const float *target,
                                                      uint32_t n, int B, int sampled, uint64_t seed,
                                                      const long long *iter_ptr, float *partial) {
  extern __shared__ float sm[];
  float *M = sm;                                 // SM_NPAR
  float *X = M + SM_NPAR;                        // [GT][NF] normalised inputs
  float *A1 = X + GT * SM_NF;                    // [GT][RS] layer-1 activations
  float *A2 = A1 + GT * RS;                      // [GT][RS] layer-2 activations
  float *D1 = A2 + GT * RS;                      // [GT][RS] layer-1 deltas
  float *D2 = D1 + GT * RS;                      // [GT][RS] layer-2 deltas
  float *DO = D2 + GT * RS;                      // [GT] output deltas
  for (int j = threadIdx.x; j < SM_NPAR; j += blockDim.x) M[j] = model[j];
  __syncthreads();
  const int t = threadIdx.x;
  const int s = blockIdx.x * GT + t;
  const long long iter = iter_ptr ? *iter_ptr : 0;
  float loss = 0.0f;
  if (s < B) {
    const uint32_t idx = sampled ? sample_index(seed, iter, s, n) : (uint32_t)s;
    float xn[SM_NF];
#pragma unroll
    for (int k = 0; k < SM_NF; k++) {
      const float v = __fmul_rn(__fsub_rn(feat[(size_t)idx * SM_NF + k], M[SM_MU + k]), M[SM_ISIG + k]);
      xn[k] = fminf(fmaxf(v, -SM_XCLAMP), SM_XCLAMP);
      X[t * SM_NF + k] = xn[k];
    }
    float a1[SM_NH];
#pragma unroll
    for (int j = 0; j < SM_NH; j++) {
      float z = M[SM_B1 + j];
#pragma unroll
      for (int k = 0; k < SM_NF; k++) z = __fmaf_rn(M[SM_W1 + j * SM_NF + k], xn[k], z);
      a1[j] = (z > 0.0f) ? z : 0.0f;
      A1[t * RS + j] = a1[j];
    }
    float out = M[SM_B3];
    for (int j = 0; j < SM_NH; j++) {
      float z = M[SM_B2 + j];
#pragma unroll
      for (int k = 0; k < SM_NH; k++) z = __fmaf_rn(M[SM_W2 + j * SM_NH + k], a1[k], z);
      z = (z > 0.0f) ? z : 0.0f;
      A2[t * RS + j] = z;
      out = __fmaf_rn(M[SM_W3 + j], z, out);
    }
    const float tn = __fdiv_rn(__fsub_rn(target[idx], M[SM_LMU]), M[SM_LSIG]);
    const float r = __fsub_rn(out, tn);
    loss = __fmul_rn(r, r);
    const float d = __fdiv_rn(__fmul_rn(2.0f, r), (float)B);
    DO[t] = d;
    float d2[SM_NH];
#pragma unroll
    for (int j = 0; j < SM_NH; j++) {
      d2[j] = (A2[t * RS + j] > 0.0f) ? __fmul_rn(d, M[SM_W3 + j]) : 0.0f;
      D2[t * RS + j] = d2[j];
    }
    for (int k = 0; k < SM_NH; k++) {
      float g = 0.0f;
#pragma unroll
      for (int j = 0; j < SM_NH; j++) g = __fmaf_rn(M[SM_W2 + j * SM_NH + k], d2[j], g);
      D1[t * RS + k] = (a1[k] > 0.0f) ? g : 0.0f;
    }
  } else {
    for (int k = 0; k < SM_NF; k++) X[t * SM_NF + k] = 0.0f;
    for (int j = 0; j < SM_NH; j++) A1[t * RS + j] = A2[t * RS + j] = D1[t * RS + j] = D2[t * RS + j] = 0.0f;
    DO[t] = 0.0f;
  }
  __syncthreads();
  // weight gradients: sums over the tile's samples in sample order
  float *out_row = partial + (size_t)blockIdx.x * PART_W;
  for (int o = t; o < SM_NTRAIN; o += GT) {
    const int j = SM_TRAIN0 + o;
    float g = 0.0f;
    if (j < SM_B1) {                      // W1[r][c]
      const int r = (j - SM_W1) / SM_NF, c = (j - SM_W1) % SM_NF;
      for (int q = 0; q < GT; q++) g = __fmaf_rn(D1[q * RS + r], X[q * SM_NF + c], g);
    } else if (j < SM_W2) {               // b1[r]
      const int r = j - SM_B1;
      for (int q = 0; q < GT; q++) g = __fadd_rn(g, D1[q * RS + r]);
    } else if (j < SM_B2) {               // W2[r][c]
      const int r = (j - SM_W2) / SM_NH, c = (j - SM_W2) % SM_NH;
      for (int q = 0; q < GT; q++) g = __fmaf_rn(D2[q * RS + r], A1[q * RS + c], g);
    } else if (j < SM_W3) {               // b2[r]
      const int r = j - SM_B2;
      for (int q = 0; q < GT; q++) g = __fadd_rn(g, D2[q * RS + r]);
    } else if (j < SM_B3) {               // W3[c]
      const int c = j - SM_W3;
      for (int q = 0; q < GT; q++) g = __fmaf_rn(DO[q], A2[q * RS + c], g);
    } else {                              // b3
      for (int q = 0; q < GT; q++) g = __fadd_rn(g, DO[q]);
    }
    out_row[o] = g;
  }
  // loss sum of the tile
  __shared__ float lred[GT];
  lred[t] = loss;
  __syncthreads();
  for (int w = GT / 2; w > 0; w >>= 1) {
    if (t < w) lred[t] = __fadd_rn(lred[t], lred[t + w]);
    __syncthreads();
  }
  if (t == 0) out_row[SM_NTRAIN] = lred[0];
}

__global__ void reduce_kernel(const float *partial, int nblk, float *grad) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < PART_W) {
    float g = 0.0f;
    for (int b = 0; b < nblk; b++) g = __fadd_rn(g, partial[(size_t)b * PART_W + o]);
    grad[o] = g;
  }
}

struct AdamState {
  float lr, b1, b2, eps;
};

// Adam step on the master weights, one block; the model's trainable block gets their
// BF16 roundings (weights) or the FP32 values (biases).  Advances the iteration counter.
__global__ void adam_kernel(float *master, float *m1, float *m2, const float *grad, float *model,
                            long long *iter_ptr, AdamState a, float *loss_hist, int hist_len) {
  const long long it = *iter_ptr;
  const float tp = (float)(it + 1);
  const float c1 = __fsub_rn(1.0f, exp_m(__fmul_rn(tp, log_m(a.b1))));
  const float c2 = __fsub_rn(1.0f, exp_m(__fmul_rn(tp, log_m(a.b2))));
  for (int o = threadIdx.x; o < SM_NTRAIN; o += blockDim.x) {
    const float g = grad[o];
    const float mm = __fmaf_rn(a.b1, m1[o], __fmul_rn(__fsub_rn(1.0f, a.b1), g));
    const float vv = __fmaf_rn(a.b2, m2[o], __fmul_rn(__fsub_rn(1.0f, a.b2), __fmul_rn(g, g)));
    m1[o] = mm;
    m2[o] = vv;
    const float step = __fdiv_rn(__fmul_rn(a.lr, __fdiv_rn(mm, c1)), __fadd_rn(__fsqrt_rn(__fdiv_rn(vv, c2)), a.eps));
    const float p = __fsub_rn(master[o], step);
    master[o] = p;
    const int j = SM_TRAIN0 + o;
    const bool w = (j >= SM_W1 && j < SM_B1) || (j >= SM_W2 && j < SM_B2) || (j >= SM_W3 && j < SM_B3);
    model[j] = w ? bf16_round(p) : p;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (loss_hist && hist_len > 0) loss_hist[it % hist_len] = grad[SM_NTRAIN];
    *iter_ptr = it + 1;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <class T> struct DevBuf {
  T *p = nullptr;
  explicit DevBuf(size_t n) { cuda_ok(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc"); }
  ~DevBuf() { if (p) cudaFree(p); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

static void set_grad_smem() {
  static bool done = false;
  if (!done) {
    cuda_ok(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GRAD_SMEM),
       "grad smem");
    done = true;
  }
}

void mlp_forward_host(const float *params, const float *feat, int n, float *out) {
  if (n <= 0) return;
  DevBuf<float> dm(SM_NPAR), df((size_t)n * SM_NF), dout(n);
  cuda_ok(cudaMemcpy(dm.p, params, SM_NPAR * sizeof(float), cudaMemcpyHostToDevice), "upload model");
  cuda_ok(cudaMemcpy(df.p, feat, (size_t)n * SM_NF * sizeof(float), cudaMemcpyHostToDevice), "upload features");
  mlp_forward_kernel<<<(n + 127) / 128, 128>>>(dm.p, df.p, n, dout.p);
  cuda_ok(cudaGetLastError(), "forward");
  cuda_ok(cudaMemcpy(out, dout.p, n * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

void mlp_grad_host(const float *params, const float *feat, const float *target, int n, float *grad,
                   float *loss) {
  if (n <= 0) throw NgpuError("empty batch");
  set_grad_smem();
  const int nblk = (n + GT - 1) / GT;
  DevBuf<float> dm(SM_NPAR), df((size_t)n * SM_NF), dt(n), part((size_t)nblk * PART_W), dg(PART_W);
  cuda_ok(cudaMemcpy(dm.p, params, SM_NPAR * sizeof(float), cudaMemcpyHostToDevice), "upload model");
  cuda_ok(cudaMemcpy(df.p, feat, (size_t)n * SM_NF * sizeof(float), cudaMemcpyHostToDevice), "upload features");
  cuda_ok(cudaMemcpy(dt.p, target, n * sizeof(float), cudaMemcpyHostToDevice), "upload targets");
  mlp_grad_kernel<<<nblk, GT, GRAD_SMEM>>>(dm.p, df.p, dt.p, (uint32_t)n, n, 0, 0, nullptr, part.p);
  reduce_kernel<<<(PART_W + 255) / 256, 256>>>(part.p, nblk, dg.p);
  cuda_ok(cudaGetLastError(), "grad");
  std::vector<float> g(PART_W);
  cuda_ok(cudaMemcpy(g.data(), dg.p, PART_W * sizeof(float), cudaMemcpyDeviceToHost), "download");
  for (int o = 0; o < SM_NTRAIN; o++) grad[o] = g[o];
  if (loss) *loss = g[SM_NTRAIN] / (float)n;
}

// He-uniform initialisation (host; deterministic in the seed).  The output layer
// starts at a tenth of that scale.
static void init_params(std::vector<float> &master, uint64_t seed) {
  auto uni = [&](uint32_t k) {   // splitmix64 of (seed, k) -> [0, 1)
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + (uint64_t)(k + 1) * 0xD1B54A32D192ED03ull;
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  master.assign(SM_NTRAIN, 0.0f);
  for (int o = 0; o < SM_NTRAIN; o++) {
    const int j = SM_TRAIN0 + o;
    double fan_in = 0;
    if (j >= SM_W1 && j < SM_B1) fan_in = SM_NF;
    else if (j >= SM_W2 && j < SM_B2) fan_in = SM_NH;
    else if (j >= SM_W3 && j < SM_B3) fan_in = SM_NH;
    if (fan_in > 0) {
      const double lim = std::sqrt(6.0 / fan_in) * ((j >= SM_W3) ? 0.1 : 1.0);
      master[o] = (float)((2.0 * uni((uint32_t)o) - 1.0) * lim);
    }
  }
}

TrainResult train_step_model(const float *d_tuples, long long n_tuples, const TrainConfig &cfg, float *params) {
  if (n_tuples <= 0) throw NgpuError("no logged RK5 steps to train on");
  set_grad_smem();
  if (n_tuples >= (1LL << 31)) throw NgpuError("too many logged RK5 steps for one training set");
  const long long n = n_tuples;
  DevBuf<int> flag(n), pos(n);
  const int fb = 148 * 8;
  tuple_flag_kernel<<<fb, 256>>>(d_tuples, n, flag.p);
  cuda_ok(cudaGetLastError(), "tuple filter");
  size_t tmp_bytes = 0;
  cuda_ok(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag.p, pos.p, (int)n), "scan size");
  DevBuf<unsigned char> tmp(tmp_bytes);
  cuda_ok(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, flag.p, pos.p, (int)n), "scan");
  int last_pos = 0, last_flag = 0;
  cuda_ok(cudaMemcpy(&last_pos, pos.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost), "count");
  cuda_ok(cudaMemcpy(&last_flag, flag.p + (n - 1), sizeof(int), cudaMemcpyDeviceToHost), "count");
  const int m = last_pos + last_flag;
  DevBuf<float> feat((size_t)std::max(m, 1) * SM_NF), tgt(std::max(m, 1));
  tuple_scatter_kernel<<<fb, 256>>>(d_tuples, n, flag.p, pos.p, feat.p, tgt.p);
  cuda_ok(cudaGetLastError(), "tuple scatter");
  TrainResult res;
  res.n_used = m;
  if (m < GT) throw NgpuError("too few logged RK5 steps where the step size is limited by accuracy (" +
                              std::to_string(m) + ")");
  // moments
  const int mb = 148 * 2;
  DevBuf<double> mom((size_t)mb * MOM_W);
  moments_kernel<<<mb, 256>>>(feat.p, tgt.p, m, mom.p);
  std::vector<double> hm((size_t)mb * MOM_W), tot(MOM_W, 0.0);
  cuda_ok(cudaMemcpy(hm.data(), mom.p, hm.size() * sizeof(double), cudaMemcpyDeviceToHost), "moments");
  for (int b = 0; b < mb; b++)
    for (int k = 0; k < MOM_W; k++) tot[k] += hm[(size_t)b * MOM_W + k];
  std::vector<float> model(SM_NPAR, 0.0f);
  for (int k = 0; k <= SM_NF; k++) {
    const double mean = tot[2 * k] / m;
    const double var = std::max(tot[2 * k + 1] / m - mean * mean, 0.0);
    const double sd = std::max(std::sqrt(var), 1e-6 * std::max(1.0, std::fabs(mean)));
    if (k < SM_NF) {
      model[SM_MU + k] = (float)mean;
      model[SM_ISIG + k] = (float)(1.0 / sd);
    } else {
      model[SM_LMU] = (float)mean;
      model[SM_LSIG] = (float)sd;
    }
  }
  model[SM_SAFETY] = cfg.safety;
  model[SM_FLOOR] = cfg.floor;
  std::vector<float> master;
  init_params(master, cfg.seed);
  for (int o = 0; o < SM_NTRAIN; o++) {
    const int j = SM_TRAIN0 + o;
    model[j] = is_weight(j) ? bf16_round_host(master[o]) : master[o];
  }
  // device training state
  const int B = std::max(GT, (cfg.batch / GT) * GT);
  const int nblk = B / GT;
  DevBuf<float> dmodel(SM_NPAR), dmaster(SM_NTRAIN), m1(SM_NTRAIN), m2(SM_NTRAIN), part((size_t)nblk * PART_W),
      grad(PART_W);
  const int hist = 64;
  DevBuf<float> loss_hist(hist);
  DevBuf<long long> iter(1);
  cuda_ok(cudaMemcpy(dmodel.p, model.data(), SM_NPAR * sizeof(float), cudaMemcpyHostToDevice), "model");
  cuda_ok(cudaMemcpy(dmaster.p, master.data(), SM_NTRAIN * sizeof(float), cudaMemcpyHostToDevice), "master");
  cuda_ok(cudaMemset(m1.p, 0, SM_NTRAIN * sizeof(float)), "m1");
  cuda_ok(cudaMemset(m2.p, 0, SM_NTRAIN * sizeof(float)), "m2");
  cuda_ok(cudaMemset(iter.p, 0, sizeof(long long)), "iter");
  cuda_ok(cudaMemset(loss_hist.p, 0, hist * sizeof(float)), "hist");
  AdamState a{cfg.lr, 0.9f, 0.999f, 1e-8f};
  cudaStream_t st;
  cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  // iterations in CUDA graphs of up to 100 iterations (the counter lives on the device)
  const int G = 100;
  cudaGraphExec_t exec = nullptr;
  int exec_len = 0;
  long long done = 0;
  try {
    while (done < cfg.iters) {
      const int len = (int)std::min<long long>(G, cfg.iters - done);
      if (!exec || exec_len != len) {
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraph_t g;
        cuda_ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
        for (int r = 0; r < len; r++) {
          mlp_grad_kernel<<<nblk, GT, GRAD_SMEM, st>>>(dmodel.p, feat.p, tgt.p, (uint32_t)m, B, 1, cfg.seed,
                                                         iter.p, part.p);
          reduce_kernel<<<(PART_W + 255) / 256, 256, 0, st>>>(part.p, nblk, grad.p);
          adam_kernel<<<1, 512, 0, st>>>(dmaster.p, m1.p, m2.p, grad.p, dmodel.p, iter.p, a,
                                                              loss_hist.p, hist);
        }
        cuda_ok(cudaStreamEndCapture(st, &g), "end capture");
        cuda_ok(cudaGraphInstantiate(&exec, g, 0), "instantiate");
        cudaGraphDestroy(g);
        exec_len = len;
      }
      cuda_ok(cudaGraphLaunch(exec, st), "train graph");
      done += len;
    }
    cuda_ok(cudaStreamSynchronize(st), "train");
  } catch (...) {
    if (exec) cudaGraphExecDestroy(exec);
    cudaStreamDestroy(st);
    throw;
  }
  if (exec) cudaGraphExecDestroy(exec);
  cudaStreamDestroy(st);
  cuda_ok(cudaMemcpy(params, dmodel.p, SM_NPAR * sizeof(float), cudaMemcpyDeviceToHost), "download model");
  std::vector<float> lh(hist);
  cuda_ok(cudaMemcpy(lh.data(), loss_hist.p, hist * sizeof(float), cudaMemcpyDeviceToHost), "loss");
  const int k = (int)std::min<long long>(hist, cfg.iters);
  double s = 0;
  for (int i = 0; i < k; i++) s += lh[i];
  res.final_loss = k > 0 ? (float)(s / k / B) : 0.0f;
  return res;
}

}  // namespace ngpu
