// NGPU_BuildDeliveryCsrNoAlloc: the delivery-layout packing of NGPU_BuildDeliveryCsr
// for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a process whose device heap
// is owned by another allocator (a PyTorch program, where the caching allocator may
// already hold most free memory, so a raw cudaMalloc can fail although the caller's
// own pool has room), or a service that carves each GPU into fixed per-tenant pools
// at start-up and forbids allocations afterwards.  Such a caller owns its input and
// output buffers but has no way to hand out scratch of a size known only inside the
// call.  This entry point takes its scratch from a file-scope device array instead,
// so it allocates nothing.
//
// Limits and sharing:
//   - the scratch holds the per-segment counters of at most NOALLOC_MAX_SEGMENTS
//     segments (n_nodes * dspan); larger problems are rejected with an error;
//   - the array is allocated when the library's device code is loaded on a GPU and
//     stays there until the process exits (about 4.3 MiB per GPU);
//   - every call shares the one array and leaves its contents behind; each call
//     clears the counters it uses before counting, so calls must not overlap on the
//     GPU (two calls on different streams at the same time race on the scratch).
//   - each call is synchronous: it waits for its work on the given stream and reads the
//     bad-index flag back before it returns;
//   - the device address of the array is looked up once per device, with that device
//     current, by the first call on it; make that first call before any stream
//     capture.
#include <cub/device/device_scan.cuh>

#include <mutex>
#include <stdexcept>
#include <string>

#include "ngpu_engine.h"
#include "ngpu_types.h"

namespace ngpu {

__global__ void list_count_kernel(size_t n, const int *src, const int *dly, int n_nodes, int dspan,
                                  unsigned long long *cnt, unsigned *bad);
__global__ void list_fill_kernel(size_t n, const int *src, const int *dly, const unsigned *target,
                                 const float *weight, int n_nodes, int dspan, unsigned long long *cursor,
                                 EdgeW *edge);

constexpr size_t NOALLOC_MAX_SEGMENTS = (size_t)1 << 19;
constexpr size_t NOALLOC_COUNTER_BYTES = (NOALLOC_MAX_SEGMENTS + 1) * sizeof(unsigned long long);
constexpr size_t NOALLOC_FLAG_OFFSET = ((NOALLOC_COUNTER_BYTES + 255) / 256) * 256;
constexpr size_t NOALLOC_SCAN_OFFSET = NOALLOC_FLAG_OFFSET + 256;
constexpr size_t NOALLOC_SCAN_BYTES = (size_t)256 << 10;
constexpr size_t NOALLOC_BYTES = NOALLOC_SCAN_OFFSET + NOALLOC_SCAN_BYTES;

// counters / cursors | bad-index flag | scan workspace
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static std::mutex g_noalloc_mutex;
static unsigned char *g_noalloc_ptr[128];   // device address of the array, per device ordinal

static unsigned char *scratch_for_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) throw std::runtime_error("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (unsigned char *)p;
  }
  return g_noalloc_ptr[dev];
}

static void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

void pack_delivery_csr_noalloc(const int *src, const int *dly, const unsigned *target, const float *weight,
                               size_t n, int n_nodes, int dspan, unsigned long long *seg_off, EdgeW *edge,
                               cudaStream_t st) {
  const size_t nkey = (size_t)n_nodes * dspan;
  if (nkey > NOALLOC_MAX_SEGMENTS)
    throw NgpuError("n_nodes * dspan = " + std::to_string(nkey) + " exceeds the " +
                    std::to_string(NOALLOC_MAX_SEGMENTS) + " segments the allocation-free scratch holds");
  unsigned char *base = scratch_for_current_device();
  unsigned long long *cnt = (unsigned long long *)base;
  unsigned *bad = (unsigned *)(base + NOALLOC_FLAG_OFFSET);
  void *scan_tmp = base + NOALLOC_SCAN_OFFSET;
  size_t scan_bytes = 0;
  ck(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt, seg_off, nkey + 1, st), "scan size");
  if (scan_bytes > NOALLOC_SCAN_BYTES) throw NgpuError("scan workspace exceeds the scratch array");
  // the array keeps the previous call's contents: clear what must start at zero
  ck(cudaMemsetAsync(cnt, 0, (nkey + 1) * sizeof(unsigned long long), st), "clear counters");
  ck(cudaMemsetAsync(bad, 0, sizeof(unsigned), st), "clear flag");
  const int gb = 148 * 8, tb = 256;
  list_count_kernel<<<gb, tb, 0, st>>>(n, src, dly, n_nodes, dspan, cnt, bad);
  ck(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, cnt, seg_off, nkey + 1, st), "scan");
  ck(cudaMemcpyAsync(cnt, seg_off, nkey * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st), "cursors");
  list_fill_kernel<<<gb, tb, 0, st>>>(n, src, dly, target, weight, n_nodes, dspan, cnt, edge);
  unsigned h_bad = 0;
  ck(cudaMemcpyAsync(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "flag");
  ck(cudaStreamSynchronize(st), "pack");
  ck(cudaGetLastError(), "pack kernels");
  if (h_bad) throw std::runtime_error("edge list holds a source or delay index out of range");
}

}  // namespace ngpu
