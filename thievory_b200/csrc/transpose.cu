// In-edge transpose of a CSR/WCSR graph, built on the device from its
// resident edge blocks: the bottom-up levels of a direction-optimising BFS
// (bfs_bottom_up in minprop.cu) scan in-edges.  The reference keeps only
// out-edges for BFS; its converter writes the same transpose as a .csc file
// (converter/converter.cpp:483-589), here it is derived in HBM instead.
//
// Two passes over the out-edges, one warp per 32 source vertices with the
// lanes striding over each list (hubs stay inside one warp): count the
// in-degree of every destination, exclusive-scan it into in_off, then
// scatter each source id into its destination's in-list.  In-list order is
// arbitrary; the BFS result does not depend on it.
#include <cub/cub.cuh>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

namespace {

struct TrArgs {
  const uint64_t *off;
  const uint32_t *blk_vb;
  const uint64_t *blk_base;
  uint32_t nblk, nv, esz, wshift;
  unsigned long long *cursor;  // in-degree counts, then fill cursors
  uint32_t *in_adj;            // null in the counting pass
};

__global__ void tr_pass(TrArgs a) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t ngroups = (a.nv + 31) / 32;
  for (uint64_t g = gwarp; g < ngroups; g += nwarps) {
    for (uint32_t j = 0; j < 32; j++) {
      const uint64_t u = g * 32 + j;
      if (u >= a.nv) break;
      const uint64_t s = __ldg(a.off + u), e = __ldg(a.off + u + 1);
      if (s == e) continue;
      const uintptr_t base = (uintptr_t)__ldg(a.blk_base + find_block(a.blk_vb, a.nblk, (uint32_t)u));
      for (uint64_t k = s + lane; k < e; k += 32) {
        const uintptr_t p = base + (uintptr_t)k * a.esz;
        const uint32_t raw = *reinterpret_cast<const uint32_t *>(p);
        const uint32_t w = a.esz == 4 ? edge_dst(raw, a.wshift) : raw;
        const unsigned long long pos = atomicAdd(a.cursor + w, 1ull);
        if (a.in_adj) a.in_adj[pos] = (uint32_t)u;
      }
    }
  }
}

__global__ void tr_copy(const unsigned long long *src, unsigned long long *dst, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

}  // namespace

void transpose_free(thv_graph *g) {
  if (g->in_valid) g->device_bytes -= (g->nv + 1) * 8 + g->ne * 4;
  dev_free(g->d_in_off);
  dev_free(g->d_in_adj);
  g->d_in_off = nullptr;
  g->d_in_adj = nullptr;
  g->in_valid = false;
}

// Needs every out-edge resident (the plan holds no host blocks).
thv_status ensure_transpose(thv_graph *g, cudaStream_t st) {
  if (g->in_valid) return THV_OK;
  if (g->fmt == THV_FMT_CSC) return fail(THV_EINVAL, "transpose of an in-edge graph");
  if (g->plan.host_edge_bytes) return fail(THV_EINVAL, "transpose needs all edges resident");
  transpose_free(g);
  const uint64_t nv = g->nv, ne = g->ne;
  THV_TRY(dev_alloc((void **)&g->d_in_off, (nv + 1) * 8 + 64, "in-edge offsets"));
  THV_TRY(dev_alloc((void **)&g->d_in_adj, ne * 4 + kEdgePad, "in-edges"));
  unsigned long long *cnt = nullptr, *cur = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  thv_status s = THV_OK;
  TrArgs a{};
  a.off = g->d_off;
  a.blk_vb = g->plan.d_vbegin;
  a.blk_base = g->plan.d_base;
  a.nblk = (uint32_t)g->plan.blocks.size();
  a.nv = (uint32_t)nv;
  a.esz = g->esz;
  a.wshift = g->wshift;
  const int grid = g->num_sms * 8;
  do {
    if ((s = dev_alloc((void **)&cnt, (nv + 1) * 8, "in-degree counts")) != THV_OK) break;
    if ((s = dev_alloc((void **)&cur, (nv + 1) * 8, "in-edge cursors")) != THV_OK) break;
    if (cudaMemsetAsync(cnt, 0, (nv + 1) * 8, st) != cudaSuccess) { s = fail(THV_ECUDA, "memset"); break; }
    a.cursor = cnt;
    a.in_adj = nullptr;
    tr_pass<<<grid, 256, 0, st>>>(a);
    // in_off = exclusive prefix sum of the counts (nv + 1 entries)
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, (unsigned long long *)g->d_in_off,
                                  (int64_t)(nv + 1), st);
    if ((s = dev_alloc(&tmp, tmp_bytes + 16, "scan scratch")) != THV_OK) break;
    if (cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, (unsigned long long *)g->d_in_off,
                                      (int64_t)(nv + 1), st) != cudaSuccess) {
      s = fail(THV_ECUDA, "in-degree scan failed");
      break;
    }
    tr_copy<<<grid, 256, 0, st>>>((const unsigned long long *)g->d_in_off, cur, nv);
    a.cursor = cur;
    a.in_adj = g->d_in_adj;
    tr_pass<<<grid, 256, 0, st>>>(a);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      s = fail(THV_ECUDA, "transpose kernels failed");
  } while (false);
  dev_free(cnt);
  dev_free(cur);
  dev_free(tmp);
  if (s != THV_OK) {
    transpose_free(g);
    return s;
  }
  g->in_valid = true;
  g->device_bytes += (nv + 1) * 8 + ne * 4;
  return THV_OK;
}

}  // namespace thv
