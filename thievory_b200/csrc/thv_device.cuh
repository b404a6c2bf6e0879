// Device-side helpers: coherent loads, warp collectives, bounded grid barrier.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "thv_internal.h"

namespace thv {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Device error codes written into a control word (0 = ok).
enum : unsigned {
  kDevOk = 0,
  kDevErrBarrier = 1,   // a grid barrier wait ran out of time
  kDevErrIters = 2,     // iteration cap reached
  kDevErrQueue = 3,     // work queue capacity exceeded
  kDevErrDepth = 4,     // batched BFS level exceeded the u8 range
};

// L2-coherent load (bypasses the non-coherent L1) for data other SMs write.
__device__ __forceinline__ uint32_t ldcg(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long ldcg(const unsigned long long *p) {
  return __ldcg(p);
}
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }

// Read-only 16-byte load; works for HBM and for host-mapped pinned memory.
__device__ __forceinline__ uint4 ld_nc_v4(uintptr_t addr) {
  return __ldg(reinterpret_cast<const uint4 *>(addr));
}
__device__ __forceinline__ uint32_t ld_nc_u32(uintptr_t addr) {
  return __ldg(reinterpret_cast<const uint32_t *>(addr));
}
__device__ __forceinline__ uint2 ld_nc_u2(uintptr_t addr) {
  return __ldg(reinterpret_cast<const uint2 *>(addr));
}

// L2 eviction priorities (createpolicy + .L2::cache_hint): streaming data
// read once (edges, queue items) is marked evict-first so that it does not
// push the randomly probed per-vertex values out of L2; those are marked
// evict-last.  A hint only orders evictions; results do not depend on it.
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_evict_last() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// Read-only 16 / 4 / 8-byte streaming loads with an L2 policy, not kept in L1.
__device__ __forceinline__ uint4 ld_stream_v4(uintptr_t addr, unsigned long long pol) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(addr), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream_u32(uintptr_t addr, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v)
               : "l"(addr), "l"(pol));
  return v;
}
__device__ __forceinline__ uint2 ld_stream_u2(uintptr_t addr, unsigned long long pol) {
  uint2 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
               : "=r"(v.x), "=r"(v.y)
               : "l"(addr), "l"(pol));
  return v;
}
// L2-coherent load / atomic min of a value other SMs write, with an L2 policy.
__device__ __forceinline__ uint32_t ldcg_hint(const uint32_t *p, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.cg.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
// atomicMin whose old value nobody waits for (a reduction).
__device__ __forceinline__ void red_min_hint(uint32_t *p, uint32_t x, unsigned long long pol) {
  asm volatile("red.global.min.L2::cache_hint.u32 [%0], %1, %2;" : : "l"(p), "r"(x), "l"(pol)
               : "memory");
}
__device__ __forceinline__ uint32_t atomic_min_hint(uint32_t *p, uint32_t x, unsigned long long pol) {
  uint32_t old;
  asm volatile("atom.global.min.L2::cache_hint.u32 %0, [%1], %2, %3;"
               : "=r"(old)
               : "l"(p), "r"(x), "l"(pol)
               : "memory");
  return old;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T x) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T y = __shfl_up_sync(kFull, x, d);
    if (lane >= (unsigned)d) x += y;
  }
  return x;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(kFull, x, d);
  return x;
}

__device__ __forceinline__ unsigned long long warp_or(unsigned long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x |= __shfl_xor_sync(kFull, x, d);
  return x;
}

__device__ __forceinline__ unsigned warp_min(unsigned x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x = min(x, __shfl_xor_sync(kFull, x, d));
  return x;
}

__device__ __forceinline__ unsigned long long shfl64(unsigned long long x,
                                                     int src) {
  return __shfl_sync(kFull, x, src);
}

// Largest lane l with excl[l] <= t, for excl non-decreasing across the warp.
__device__ __forceinline__ int warp_owner(unsigned excl, unsigned t) {
  int pos = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const unsigned e = __shfl_sync(kFull, excl, pos + s);
    if (e <= t) pos += s;
  }
  return pos;
}

// Frontier work item: the adjacency of vertex v (or one chunk of it) at a
// device or host-mapped address.
struct __align__(16) WorkItem {
  uint64_t eaddr;
  uint32_t v;
  uint32_t cnt;
};

constexpr uint32_t kSmemBlocks = 2048;  // block tables up to this size go to smem

// Edge block of vertex v: largest b with vb[b] <= v (vb has nblk+1 entries).
__device__ __forceinline__ uint32_t find_block(const uint32_t *vb, uint32_t nblk,
                                               uint32_t v) {
  uint32_t lo = 0, hi = nblk;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (vb[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// A 4-byte edge: the neighbour id in the high bits and, for packed weighted
// graphs, w - wbase in the low wshift bits (wshift = 0: an id-only edge).
__device__ __forceinline__ uint32_t edge_dst(uint32_t e, uint32_t wshift) { return e >> wshift; }
__device__ __forceinline__ uint32_t edge_wt(uint32_t e, uint32_t wshift, uint32_t wbase) {
  return (e & ((1u << wshift) - 1u)) + wbase;
}

// Device address of the first edge of v's list, given its block's base and
// its first edge index s0; *host says whether it is read over the host link.
__device__ __forceinline__ unsigned long long list_addr(const ListCache &lc,
                                                       unsigned long long block_base,
                                                       unsigned long long host_base, uint32_t v,
                                                       uint64_t s0, uint32_t deg, uint32_t esz,
                                                       bool *host) {
  const bool on_host = block_base == host_base;
  if (on_host && deg < lc.deg_lt && deg > 0) {
    *host = false;
    return lc.base + (unsigned long long)__ldg(lc.idx + v) * esz;
  }
  *host = on_host;
  return block_base + s0 * esz;
}

// Grid-wide barrier for a cooperative launch.  The wait is bounded by
// timeout_ns of %globaltimer; on expiry the error word is set and every
// block leaves through the false return.  Returns false if any block has
// flagged an error.
struct GridBar {
  unsigned count;
  unsigned gen;
};

__device__ __forceinline__ bool grid_sync(GridBar *bar, unsigned *err,
                                          unsigned long long timeout_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned gen = *((volatile unsigned *)&bar->gen);
    __threadfence();
    const unsigned arrived = atomicAdd(&bar->count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned spins = 0;
      while (*((volatile unsigned *)&bar->gen) == gen) {
        if ((++spins & 63u) == 0 && global_ns() - t0 > timeout_ns) {
          atomicCAS(err, 0u, kDevErrBarrier);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *((volatile unsigned *)err) == 0;
}

}  // namespace thv
