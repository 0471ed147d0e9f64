// Learned RK5 step-size proposal: the logging / proposing variants of the aeif
// kernels and the MLP kernels that train the proposal network on the GPU.
//
// Training (per iteration, minibatch of B sampled tuples):
//   mlp_grad_kernel    one 128-sample tile per block: the layer products, the
//                      back-propagated error product and one product for all weight
//                      and bias gradients (dW = sum_s delta_s a_s^T) on the tensor
//                      cores (tcgen05, BF16 operands, FP32 accumulators in tensor
//                      memory); one thread per sample for the elementwise work; one
//                      partial gradient row per block;
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
// gradient of the mean squared error over one tile of 128 samples per block, on the
// tensor cores: tcgen05.mma with BF16 operands in shared memory and FP32 accumulators in
// tensor memory (TMEM), issued by one thread; the elementwise work between the products
// (biases, ReLU, the output layer, the loss) runs on the CUDA cores, one thread per sample.
//
//   Z1 = X . W1^T       X [128 x 16] . W1^T            -> TMEM columns   0..31
//   Z2 = A1 . W2^T      A1 [128 x 32] . W2^T           -> TMEM columns  32..63
//   G1 = D2 . W2        D2 [128 x 32] . (W2^T)^T       -> TMEM columns  64..95
//   one product for every weight and bias gradient (K = the 128 samples):
//     GA [128 x 128] = rows D2^T (0..31), D1^T (32..63), d^T (64), zeros
//     GB [ 96 x 128] = rows A1^T (0..31), A2^T (32..63), X^T (64..73), ones (80), zeros
//     GA . GB^T -> TMEM columns 96..191: dW2 = rows 0..31 x cols 0..31, dW1 = rows 32..63 x
//     cols 64..73, dW3 = row 64 x cols 32..63, and the bias gradients in col 80.
// Operand precision: the inputs, activations and back-propagated errors enter the products
// as BF16 roundings (the weights are BF16 values already); sums are FP32.
// ---------------------------------------------------------------------------
constexpr int GT = 128;                  // samples per tile = threads per block = MMA M
constexpr int PART_W = SM_NTRAIN + 1;    // partial row: gradients, then the loss sum

// Byte offset of element (r, k) of a BF16 operand tile with K columns, in the K-major
// no-swizzle layout of the tensor core's shared-memory descriptors: 8-row x 16-byte core
// matrices, the K-chunks of an 8-row group adjacent (128 B apart: the descriptor's leading
// byte offset), the 8-row groups K/8 x 128 B apart (its stride byte offset).
__host__ __device__ constexpr int tile_off(int r, int k, int K) {
  return (r >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}
constexpr int TC_X = 0;                          // [128 x 16]
constexpr int TC_W1 = TC_X + 128 * 16 * 2;       // [ 32 x 16]  W1[j][k]
constexpr int TC_A1 = TC_W1 + 32 * 16 * 2;       // [128 x 32]
constexpr int TC_W2 = TC_A1 + 128 * 32 * 2;      // [ 32 x 32]  W2[j][k]
constexpr int TC_D2 = TC_W2 + 32 * 32 * 2;       // [128 x 32]
constexpr int TC_W2T = TC_D2 + 128 * 32 * 2;     // [ 32 x 32]  W2[k][j] at (j, k)
constexpr int TC_GA = TC_W2T + 32 * 32 * 2;      // [128 x 128]
constexpr int TC_GB = TC_GA + 128 * 128 * 2;     // [ 96 x 128]
constexpr int TC_M = TC_GB + 96 * 128 * 2;       // model parameters (floats)
// (the 8 KB tail keeps every address a descriptor can form from these tiles inside the
// block's shared memory)
constexpr size_t GRAD_SMEM = TC_M + sizeof(float) * SM_NPAR + 8192;
constexpr int TC_COLS = 256;                     // TMEM columns allocated (192 used)
constexpr long long TC_WAIT_POLLS = 1LL << 22;   // bound of each wait for the tensor core

// Shared-memory matrix descriptor of a K-major no-swizzle tile with K columns whose first
// K-chunk starts at shared address `addr`: start >> 4 (bits 0-13), leading byte offset
// 128 >> 4 (bits 16-29), stride byte offset (K/8 * 128) >> 4 (bits 32-45), descriptor
// version 1 (bits 46-47), base offset 0, layout "no swizzle" (bits 61-63 = 0).
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, int K) {
  return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(((K / 8) * 128) >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B
// (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 (bits 17-22), M >> 4
// (bits 24-28).
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// D[128 x N] (+)= A[128 x K] . B[N x K]^T, K/16 instructions; issued by one thread.
__device__ __forceinline__ void tc_gemm(uint32_t d_tmem, uint32_t a, uint32_t b, int K, uint32_t idesc) {
  for (int s = 0; s < K / 16; s++) {
    const uint64_t ad = tc_desc(a + 256u * s, K), bd = tc_desc(b + 256u * s, K);
    const uint32_t acc = s > 0 ? 1u : 0u;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 ::"r"(d_tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
  }
}
// The barrier's phase completes when the MMAs this thread issued before are done.
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
// Waits for phase `parity` of the barrier, at most `polls` polls; false if it gave up.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, long long polls) {
  for (long long i = 0; i < polls; i++) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive TMEM columns of this thread's lane (warp w reads lanes 32w .. 32w+31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t bf16_bits(float v) {
  bool sp;
  return __float_as_uint(bf16_round_bits(__float_as_uint(v), sp)) >> 16;
}
// Row t of a K-major tile from K floats (rounded to BF16), one 16-byte store per 8 values.
template <int K>
__device__ __forceinline__ void put_row(unsigned char *tile, int t, const float *v) {
#pragma unroll
  for (int c = 0; c < K / 8; c++) {
    uint4 q;
    q.x = bf16_bits(v[8 * c + 0]) | (bf16_bits(v[8 * c + 1]) << 16);
    q.y = bf16_bits(v[8 * c + 2]) | (bf16_bits(v[8 * c + 3]) << 16);
    q.z = bf16_bits(v[8 * c + 4]) | (bf16_bits(v[8 * c + 5]) << 16);
    q.w = bf16_bits(v[8 * c + 6]) | (bf16_bits(v[8 * c + 7]) << 16);
    *reinterpret_cast<uint4 *>(tile + tile_off(t, 8 * c, K)) = q;
  }
}
// Column t (a sample) of rows r0 .. r0+n-1 of a tile with K = 128 columns.
__device__ __forceinline__ void put_col(unsigned char *tile, int r0, int n, int t, const float *v) {
  for (int i = 0; i < n; i++)
    *reinterpret_cast<unsigned short *>(tile + tile_off(r0 + i, t, GT)) = (unsigned short)bf16_bits(v[i]);
}

__device__ __forceinline__ uint32_t sample_index(uint64_t seed, long long iter, int s, uint32_t n) {
  U4 c{(uint32_t)s, (uint32_t)iter, (uint32_t)((unsigned long long)iter >> 32), 0x51ed2701u};
  U4 r = philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return (uint32_t)(((unsigned long long)r.x * n) >> 32);
}

// Samples: tile blockIdx.x covers batch positions [GT*blockIdx.x, GT*blockIdx.x+GT) of B;
// position s uses sample sample_index(seed, iter, s) if sampled, else sample s.  Positions
// past B contribute nothing (their output error is zero).  A wait for the tensor core that
// gives up sets bit 0 of *status and the block ends after releasing its TMEM.  test_no_commit
// (failure-path test only): the products are issued but their completion is never signalled,
// so the first wait runs out after a short bound.
__global__ void __launch_bounds__(GT) mlp_grad_kernel(const float *model, const float *feat, const float *target,
                                                      uint32_t n, int B, int sampled, uint64_t seed,
                                                      const long long *iter_ptr, float *partial,
                                                      unsigned *status, int test_no_commit) {
  extern __shared__ __align__(128) unsigned char tc_sm[];
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ uint32_t s_taddr;
  __shared__ int s_fail;
  __shared__ float lred[GT];
  float *M = reinterpret_cast<float *>(tc_sm + TC_M);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t bar = smem_u32(&s_bar);
  // zero the gradient operands (their padding rows stay zero), load the model
  {
    uint4 *z = reinterpret_cast<uint4 *>(tc_sm + TC_GA);
    const int nz = (TC_M - TC_GA) / 16;
    for (int i = t; i < nz; i += GT) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (int j = t; j < SM_NPAR; j += GT) M[j] = model[j];
  if (t == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                 "r"(TC_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = s_taddr;
  const uint32_t my_lanes = tm + ((uint32_t)(warp * 32) << 16);
  unsigned char *S = tc_sm;
  // weight operands
  for (int e = t; e < 32 * 16; e += GT) {
    const int j = e / 16, k = e % 16;
    const float w = k < SM_NF ? M[SM_W1 + j * SM_NF + k] : 0.0f;
    *reinterpret_cast<unsigned short *>(S + TC_W1 + tile_off(j, k, 16)) = (unsigned short)bf16_bits(w);
  }
  for (int e = t; e < 32 * 32; e += GT) {
    const int j = e / 32, k = e % 32;
    const unsigned short w = (unsigned short)bf16_bits(M[SM_W2 + j * SM_NH + k]);
    *reinterpret_cast<unsigned short *>(S + TC_W2 + tile_off(j, k, 32)) = w;
    *reinterpret_cast<unsigned short *>(S + TC_W2T + tile_off(k, j, 32)) = w;
  }
  __syncthreads();
  // layer 1 input
  const int s = blockIdx.x * GT + t;
  const bool valid = s < B;
  const long long iter = iter_ptr ? *iter_ptr : 0;
  uint32_t idx = 0;
  float xn[16];
#pragma unroll
  for (int k = 0; k < 16; k++) xn[k] = 0.0f;
  if (valid) {
    idx = sampled ? sample_index(seed, iter, s, n) : (uint32_t)s;
#pragma unroll
    for (int k = 0; k < SM_NF; k++) {
      const float v = __fmul_rn(__fsub_rn(feat[(size_t)idx * SM_NF + k], M[SM_MU + k]), M[SM_ISIG + k]);
      xn[k] = fminf(fmaxf(v, -SM_XCLAMP), SM_XCLAMP);
    }
  }
  put_row<16>(S + TC_X, t, xn);
  put_col(S + TC_GB, 64, SM_NF, t, xn);
  {
    const float one = 1.0f;
    put_col(S + TC_GB, 80, 1, t, &one);
  }
  float loss = 0.0f;
  uint32_t phase = 0;
  // the four products, each followed by its epilogue
  float a1[SM_NH], z[32];
  for (int stage = 0; stage < 4; stage++) {
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      if (stage == 0) tc_gemm(tm + 0, smem_u32(S + TC_X), smem_u32(S + TC_W1), 16, tc_idesc(128, 32));
      else if (stage == 1) tc_gemm(tm + 32, smem_u32(S + TC_A1), smem_u32(S + TC_W2), 32, tc_idesc(128, 32));
      else if (stage == 2) tc_gemm(tm + 64, smem_u32(S + TC_D2), smem_u32(S + TC_W2T), 32, tc_idesc(128, 32));
      else tc_gemm(tm + 96, smem_u32(S + TC_GA), smem_u32(S + TC_GB), GT, tc_idesc(128, 96));
      if (!test_no_commit) tc_commit(bar);
    }
    const bool ok = tc_wait(bar, phase, test_no_commit ? (1LL << 12) : TC_WAIT_POLLS);
    phase ^= 1u;
    if (!ok) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    tc_fence_after();
    if (stage == 0) {
      tmem_ld32(my_lanes + 0, z);
#pragma unroll
      for (int j = 0; j < SM_NH; j++) {
        const float v = __fadd_rn(z[j], M[SM_B1 + j]);
        a1[j] = (valid && v > 0.0f) ? v : 0.0f;
      }
      put_row<32>(S + TC_A1, t, a1);
      put_col(S + TC_GB, 0, SM_NH, t, a1);
    } else if (stage == 1) {
      tmem_ld32(my_lanes + 32, z);
      float a2[SM_NH];
      float out = M[SM_B3];
#pragma unroll
      for (int j = 0; j < SM_NH; j++) {
        const float v = __fadd_rn(z[j], M[SM_B2 + j]);
        a2[j] = (valid && v > 0.0f) ? v : 0.0f;
        out = __fmaf_rn(M[SM_W3 + j], a2[j], out);
      }
      put_col(S + TC_GB, 32, SM_NH, t, a2);
      float d = 0.0f;
      if (valid) {
        const float tn = __fdiv_rn(__fsub_rn(target[idx], M[SM_LMU]), M[SM_LSIG]);
        const float r = __fsub_rn(out, tn);
        loss = __fmul_rn(r, r);
        d = __fdiv_rn(__fmul_rn(2.0f, r), (float)B);
      }
      float d2[SM_NH];
#pragma unroll
      for (int j = 0; j < SM_NH; j++) d2[j] = (a2[j] > 0.0f) ? __fmul_rn(d, M[SM_W3 + j]) : 0.0f;
      put_row<32>(S + TC_D2, t, d2);
      put_col(S + TC_GA, 0, SM_NH, t, d2);
      put_col(S + TC_GA, 64, 1, t, &d);
    } else if (stage == 2) {
      tmem_ld32(my_lanes + 64, z);
      float d1[SM_NH];
#pragma unroll
      for (int k = 0; k < SM_NH; k++) d1[k] = (a1[k] > 0.0f) ? z[k] : 0.0f;
      put_col(S + TC_GA, 32, SM_NH, t, d1);
    } else {
      // gradients: warp 0 holds rows 0..31 (W2, b2), warp 1 rows 32..63 (W1, b1), lane 0 of
      // warp 2 row 64 (W3, b3)
      float *out_row = partial + (size_t)blockIdx.x * PART_W;
      float g[32], gb[16];
      if (warp == 0) {
        tmem_ld32(my_lanes + 96, g);
        tmem_ld16(my_lanes + 96 + 80, gb);
#pragma unroll
        for (int c = 0; c < SM_NH; c++) out_row[SM_W2 - SM_TRAIN0 + lane * SM_NH + c] = g[c];
        out_row[SM_B2 - SM_TRAIN0 + lane] = gb[0];
      } else if (warp == 1) {
        tmem_ld32(my_lanes + 96 + 64, g);
#pragma unroll
        for (int k = 0; k < SM_NF; k++) out_row[SM_W1 - SM_TRAIN0 + lane * SM_NF + k] = g[k];
        out_row[SM_B1 - SM_TRAIN0 + lane] = g[16];
      } else if (warp == 2) {
        tmem_ld32(my_lanes + 96 + 32, g);
        tmem_ld16(my_lanes + 96 + 80, gb);
        if (lane == 0) {
#pragma unroll
          for (int c = 0; c < SM_NH; c++) out_row[SM_W3 - SM_TRAIN0 + c] = g[c];
          out_row[SM_B3 - SM_TRAIN0] = gb[0];
        }
      }
    }
  }
  if (s_fail) {
    // a product did not complete in time: record it and wait once more (bounded) for the
    // tensor core before the TMEM is released
    if (t == 0) {
      atomicOr(status, 1u);
      if (!test_no_commit) tc_wait(bar, phase ^ 1u, TC_WAIT_POLLS);
    }
  }
  // loss sum of the tile
  lred[t] = loss;
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TC_COLS) : "memory");
  for (int w = GT / 2; w > 0; w >>= 1) {
    if (t < w) lred[t] = __fadd_rn(lred[t], lred[t + w]);
    __syncthreads();
  }
  if (t == 0 && !s_fail) partial[(size_t)blockIdx.x * PART_W + SM_NTRAIN] = lred[0];
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

// Test hook of the training kernel's failure path (mlp_grad_kernel's test_no_commit).
static int g_test_no_commit = 0;
void set_tensor_wait_test(int on) { g_test_no_commit = on ? 1 : 0; }

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
  DevBuf<unsigned> st(1);
  cuda_ok(cudaMemset(st.p, 0, sizeof(unsigned)), "status");
  cuda_ok(cudaMemcpy(dm.p, params, SM_NPAR * sizeof(float), cudaMemcpyHostToDevice), "upload model");
  cuda_ok(cudaMemcpy(df.p, feat, (size_t)n * SM_NF * sizeof(float), cudaMemcpyHostToDevice), "upload features");
  cuda_ok(cudaMemcpy(dt.p, target, n * sizeof(float), cudaMemcpyHostToDevice), "upload targets");
  mlp_grad_kernel<<<nblk, GT, GRAD_SMEM>>>(dm.p, df.p, dt.p, (uint32_t)n, n, 0, 0, nullptr, part.p, st.p,
                                           g_test_no_commit);
  reduce_kernel<<<(PART_W + 255) / 256, 256>>>(part.p, nblk, dg.p);
  cuda_ok(cudaGetLastError(), "grad");
  unsigned hst = 0;
  cuda_ok(cudaMemcpy(&hst, st.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
  if (hst) throw NgpuError("MLP gradient: a tensor-core product did not complete");
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
  DevBuf<unsigned> status(1);
  cuda_ok(cudaMemset(status.p, 0, sizeof(unsigned)), "status");
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
                                                         iter.p, part.p, status.p, g_test_no_commit);
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
  unsigned hst = 0;
  cuda_ok(cudaMemcpy(&hst, status.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
  if (hst) throw NgpuError("step model training: a tensor-core product did not complete");
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
