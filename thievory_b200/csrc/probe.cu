// Host-link bandwidth probe: the denominator for zero-copy edge reads.
#include <algorithm>
#include <cstring>

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
