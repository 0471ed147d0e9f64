// Measured denominator for the delivery kernel's roofline: the rate of FP64 reductions
// (red.global.add.f64) to uniformly random addresses of a buffer, the access pattern of the
// delivery's accumulator updates (random targets inside one accumulator slot).  No
// counterpart in the reference.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace ngpu {

__global__ void random_reduction_kernel(double *buf, unsigned long long n_elem, long long ops_per_thread,
                                        unsigned seed) {
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  unsigned x = (unsigned)(tid * 2654435761ULL) ^ seed;
  for (long long k = 0; k < ops_per_thread; k++) {
    // xorshift32: a new pseudo-random index per operation
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    atomicAdd(&buf[x % n_elem], 1.0);
  }
}

static void probe_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// Reductions per second (1e9) over a buffer of `bytes` bytes, `n_ops` reductions in total
// (after one untimed launch of the same size).
double measure_random_reduction_rate(size_t bytes, long long n_ops) {
  const unsigned long long n_elem = bytes / sizeof(double);
  if (n_elem < 1 || n_ops < 1) throw std::runtime_error("reduction probe: empty buffer or no operations");
  int dev = 0, n_sm = 0;
  probe_ok(cudaGetDevice(&dev), "device");
  probe_ok(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev), "attribute");
  const int threads = 256, blocks = n_sm * 8;
  const long long per = (n_ops + (long long)threads * blocks - 1) / ((long long)threads * blocks);
  double *buf = nullptr;
  probe_ok(cudaMalloc(&buf, n_elem * sizeof(double)), "cudaMalloc");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float ms = 0.0f;
  cudaError_t err = cudaMemset(buf, 0, n_elem * sizeof(double));
  if (err == cudaSuccess) {
    random_reduction_kernel<<<blocks, threads>>>(buf, n_elem, per, 12345u);
    cudaEventRecord(a);
    random_reduction_kernel<<<blocks, threads>>>(buf, n_elem, per, 67890u);
    cudaEventRecord(b);
    err = cudaEventSynchronize(b);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, a, b);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  probe_ok(err, "reduction probe");
  return (double)per * threads * blocks / (ms * 1e-3) / 1e9;
}

}  // namespace ngpu
