// Host-link bandwidth probe: the denominator for zero-copy edge reads.
#include <algorithm>
#include <cstring>
#include <exception>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

// Streams `n16` 16-byte words from host-mapped memory, the same load the
// engine uses for non-resident edge blocks; folds them so the loads stay.
__global__ void zero_copy_stream(uintptr_t base, uint64_t n16, uint32_t *sink) {
  uint32_t acc = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 q = ld_nc_v4(base + 16 * i);
    acc ^= q.x ^ q.y ^ q.z ^ q.w;
  }
  if (acc == 0x9E3779B9u) sink[0] = acc;  // practically never; keeps the loads
}

static thv_status measure(int device, uint64_t bytes, double *mc, double *zc) {
  THV_CUDA(cudaSetDevice(device));
  bytes = std::max<uint64_t>(bytes, 1 << 20) / 16 * 16;
  void *h = nullptr, *d = nullptr;
  THV_TRY(pinned_alloc(&h, bytes, "probe host buffer"));
  thv_status s = dev_alloc(&d, bytes, "probe device buffer");
  if (s != THV_OK) { pinned_free(h); return s; }
  memset(h, 1, bytes);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_mc = 1e30f, best_zc = 1e30f;
  void *hd = nullptr;
  cudaHostGetDevicePointer(&hd, h, 0);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep) best_mc = std::min(best_mc, ms);
    cudaEventRecord(e0);
    zero_copy_stream<<<prop.multiProcessorCount * 8, 256>>>((uintptr_t)hd, bytes / 16, (uint32_t *)d);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep) best_zc = std::min(best_zc, ms);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(d);
  pinned_free(h);
  if (err != cudaSuccess) return fail(THV_ECUDA, "link probe: %s", cudaGetErrorString(err));
  if (mc) *mc = bytes / (best_mc * 1e-3) / 1e9;
  if (zc) *zc = bytes / (best_zc * 1e-3) / 1e9;
  return THV_OK;
}

}  // namespace thv

extern "C" thv_status thv_link_bandwidth(int device, uint64_t bytes, double *memcpy_gbs,
                                         double *zerocopy_gbs) {
  try {
    return thv::measure(device, bytes, memcpy_gbs, zerocopy_gbs);
  } catch (...) {
    return thv::fail(THV_EINVAL, "exception in link probe");
  }
}

// ---------------------------------------------------------- wait timeout --
// Block 0 leaves without reaching the grid barrier, so block 1's bounded
// wait runs out after timeout_ns and records the barrier error: the path a
// traversal takes when a block stops making progress, exercised without a
// fault (the wait is limited by %globaltimer and always ends).
namespace thv {

__global__ void wait_timeout_probe(GridBar *bar, unsigned *err, unsigned long long timeout_ns) {
  if (blockIdx.x == 0) return;
  grid_sync(bar, err, timeout_ns);
}

}  // namespace thv

extern "C" thv_status thv_debug_wait_timeout(int device, uint32_t timeout_ms) {
  using namespace thv;
  try {
    if (timeout_ms == 0 || timeout_ms > 10000) return fail(THV_EINVAL, "timeout must be 1..10000 ms");
    THV_CUDA(cudaSetDevice(device));
    struct Scratch {
      GridBar bar;
      unsigned err, pad;
    };
    Scratch *d = nullptr;
    THV_TRY(dev_alloc((void **)&d, sizeof(Scratch), "wait probe"));
    Scratch h{};
    thv_status s = THV_OK;
    if (cudaMemset(d, 0, sizeof(Scratch)) != cudaSuccess) s = fail(THV_ECUDA, "memset");
    if (s == THV_OK) {
      wait_timeout_probe<<<2, 32>>>(&d->bar, &d->err, (unsigned long long)timeout_ms * 1000000ull);
      if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
          cudaMemcpy(&h, d, sizeof(Scratch), cudaMemcpyDeviceToHost) != cudaSuccess)
        s = fail(THV_ECUDA, "wait probe launch failed");
    }
    dev_free(d);
    if (s != THV_OK) return s;
    if (h.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "grid barrier wait exceeded %u ms", timeout_ms);
    return fail(THV_EDEVICE, "wait probe ended without a timeout (error word %u)", h.err);
  } catch (const std::exception &e) {
    return fail(THV_ECUDA, "wait probe: %s", e.what());
  }
}
