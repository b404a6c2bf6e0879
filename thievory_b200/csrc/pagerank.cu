// PageRank, pull (CSC in-edges) and push (CSR out-edges).
//
// Method (fixed by the engine's contract, not the reference's): FP32 ranks,
// damping d, a fixed iteration count, dangling mass spread uniformly:
//     r'(v) = (1-d)/N + d * ( sum_{u->v} r(u)/outdeg(u) + D/N ),
//     D = sum of r(u) over vertices with outdeg(u) = 0,   r0 = 1/N.
// The reference's kernels this replaces are src/pr/pr_kernels.cu:23-160
// (pull: static/demand/filter) with PR32_Update_Values :449-476, and
// :504-681 (push) with PR32_Update_Values_PUSH :846-860; those iterate to a
// 1e-3 tolerance in FP64 without dangling redistribution.
//
// Every iteration streams all edges.  A CTA takes one tile (<= 4096 edges of
// consecutive vertices inside one edge block), stages the tile's adjacency in
// shared memory with 16-byte vector loads -- full 128-byte lines whether the
// block is in HBM or read zero-copy from pinned host memory -- and then
// gathers (pull) or scatters (push) per edge.  Per-vertex sums are FP64
// (warp segmented reductions); stored ranks and contributions are FP32.
// Pull fuses the rank update into the gather: a vertex's sum is complete
// inside its tile, except high-degree vertices cut into parts, whose last
// part (atomic counter) finishes the update.
#include <algorithm>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

constexpr int kPrThreads = 256;
constexpr int kPrWarps = kPrThreads / 32;
constexpr int kStageEdges = 4096;  // == kTileEdges of the tiler

struct PrArgs {
  const PrTile *tiles;
  const uint64_t *blk_base;
  const uint64_t *off;
  const uint32_t *outdeg;  // CSC: explicit; CSR: nullptr (from offsets)
  const float *cur;
  float *nxt;
  float *rank;
  double *sum;
  double *split_acc;
  uint32_t *split_done;
  const uint32_t *split_parts;
  double *dang;
  uint32_t *tile_ctr;
  uint32_t ntiles, nv, it;
  uint32_t wshift;  // packed weighted edges: the id is e >> wshift
  double damping, inv_n;
};

struct PrState {
  uint64_t nv = 0;
  uint32_t iters = 0;
  float *d_c[2] = {nullptr, nullptr};
  float *d_rank = nullptr;
  double *d_sum = nullptr;
  double *d_split_acc = nullptr;
  uint32_t *d_split_done = nullptr;
  double *d_dang = nullptr;
  uint32_t *d_tile_ctr = nullptr;
  uint32_t cap_iters = 0;
  size_t nsplit = 0;
  bool push = false;
  // reference semantics (THV_RUN_PR_REFERENCE): FP64 values
  bool ref = false;
  double *d_val = nullptr, *d_acc = nullptr, *d_delta = nullptr;
  uint8_t *d_act = nullptr;
  unsigned long long *d_cnt = nullptr, *h_cnt = nullptr;  // active vertices, their edges
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

__device__ __forceinline__ uint32_t out_degree(const PrArgs &a, uint32_t v) {
  return a.outdeg ? __ldg(a.outdeg + v)
                  : (uint32_t)(__ldg(a.off + v + 1) - __ldg(a.off + v));
}

__device__ __forceinline__ double finish_vertex(const PrArgs &a, uint32_t v,
                                                double sum, double base) {
  const double r = base + a.damping * sum;
  a.rank[v] = (float)r;
  const uint32_t od = out_degree(a, v);
  a.nxt[v] = od ? (float)(r / (double)od) : 0.f;
  return od ? 0.0 : r;
}

template <int ESZ>
__device__ __forceinline__ uint32_t staged_id(const uint32_t *s_e, uint32_t i, uint32_t wshift) {
  return ESZ == 4 ? edge_dst(s_e[i], wshift) : s_e[(size_t)i * 2];
}

// Stage edges [t.ebegin, t.eend) of a tile; returns the element shift.
template <int ESZ>
__device__ __forceinline__ uint32_t stage_tile(const PrArgs &a, const PrTile &t,
                                               uint32_t *s_e) {
  const uintptr_t b = (uintptr_t)__ldg(a.blk_base + t.block);
  const uintptr_t s0 = b + (uintptr_t)t.ebegin * ESZ;
  const uintptr_t s1 = b + (uintptr_t)t.eend * ESZ;
  const uintptr_t a0 = s0 & ~(uintptr_t)15;
  const uint32_t nvec = (uint32_t)((s1 - a0 + 15) / 16);
  uint4 *dst = reinterpret_cast<uint4 *>(s_e);
  for (uint32_t i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = ld_nc_v4(a0 + 16u * i);
  return (uint32_t)((s0 - a0) / ESZ);
}

__device__ __forceinline__ double block_sum(double x, double *s_red) {
  x = warp_sum(x);
  const unsigned w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) s_red[w] = x;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (unsigned)kPrWarps ? s_red[threadIdx.x] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;  // valid in thread 0..31
}

template <int ESZ>
__global__ void __launch_bounds__(kPrThreads) pr_pull_kernel(PrArgs a) {
  __shared__ __align__(16) uint32_t s_e[kStageEdges * (ESZ / 4) + 16];
  __shared__ double s_acc[kPrWarps][32];
  __shared__ double s_red[kPrWarps];
  __shared__ uint32_t s_tile;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  const double base = (1.0 - a.damping) * a.inv_n + a.damping * ldcg(a.dang + a.it) * a.inv_n;
  double dsum = 0.0;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr + a.it, 1u);
    __syncthreads();
    const uint32_t ti = s_tile;
    if (ti >= a.ntiles) break;
    const PrTile t = a.tiles[ti];
    const uint32_t shift = stage_tile<ESZ>(a, t, s_e);
    __syncthreads();
    if (t.split) {
      const uint32_t cnt = (uint32_t)(t.eend - t.ebegin);
      double part = 0.0;
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
        part += (double)__ldg(a.cur + staged_id<ESZ>(s_e, shift + i, a.wshift));
      part = block_sum(part, s_red);
      if (threadIdx.x == 0) {
        const uint32_t s = t.split - 1;
        atomicAdd(a.split_acc + s, part);
        __threadfence();
        const uint32_t done = atomicAdd(a.split_done + s, 1u);
        if (done + 1 == __ldg(a.split_parts + s)) {
          __threadfence();
          const unsigned long long bits =
              atomicExch(reinterpret_cast<unsigned long long *>(a.split_acc + s), 0ull);
          a.split_done[s] = 0;
          dsum += finish_vertex(a, t.vbegin, __longlong_as_double((long long)bits), base);
        }
      }
    } else {
      const uint32_t nverts = t.vend - t.vbegin;
      const uint32_t ngroups = (nverts + 31) / 32;
      for (uint32_t g = warp; g < ngroups; g += kPrWarps) {
        const uint32_t v = t.vbegin + g * 32 + lane;
        const bool valid = v < t.vend;
        uint32_t ls = 0, deg = 0;
        if (valid) {
          const uint64_t e0 = __ldg(a.off + v), e1 = __ldg(a.off + v + 1);
          ls = (uint32_t)(e0 - t.ebegin);
          deg = (uint32_t)(e1 - e0);
        }
        const unsigned incl = warp_incl_scan<unsigned>(deg);
        const unsigned excl = incl - deg;
        const unsigned total = __shfl_sync(kFull, incl, 31);
        s_acc[warp][lane] = 0.0;
        __syncwarp();
        for (unsigned k = 0; k < total; k += 32) {
          const unsigned tt = k + lane;
          const int o = warp_owner(excl, tt);
          const unsigned ols = __shfl_sync(kFull, ls, o);
          const unsigned oex = __shfl_sync(kFull, excl, o);
          double x = 0.0;
          int pos = 32;
          if (tt < total) {
            x = (double)__ldg(a.cur + staged_id<ESZ>(s_e, shift + ols + (tt - oex), a.wshift));
            pos = o;
          }
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_up_sync(kFull, x, d);
            const int pp = __shfl_up_sync(kFull, pos, d);
            if (lane >= (unsigned)d && pp == pos) x += y;
          }
          const int nxt = __shfl_down_sync(kFull, pos, 1);
          if ((lane == 31 || nxt != pos) && pos < 32) s_acc[warp][pos] += x;
          __syncwarp();
        }
        if (valid) dsum += finish_vertex(a, v, s_acc[warp][lane], base);
        __syncwarp();
      }
    }
    __syncthreads();
  }
  dsum = block_sum(dsum, s_red);
  if (threadIdx.x == 0 && dsum != 0.0) atomicAdd(a.dang + a.it + 1, dsum);
}

template <int ESZ>
__global__ void __launch_bounds__(kPrThreads) pr_push_kernel(PrArgs a) {
  __shared__ __align__(16) uint32_t s_e[kStageEdges * (ESZ / 4) + 16];
  __shared__ uint32_t s_tile;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr + a.it, 1u);
    __syncthreads();
    const uint32_t ti = s_tile;
    if (ti >= a.ntiles) break;
    const PrTile t = a.tiles[ti];
    const uint32_t shift = stage_tile<ESZ>(a, t, s_e);
    __syncthreads();
    if (t.split) {
      const double c = (double)__ldg(a.cur + t.vbegin);
      const uint32_t cnt = (uint32_t)(t.eend - t.ebegin);
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
        atomicAdd(a.sum + staged_id<ESZ>(s_e, shift + i, a.wshift), c);
    } else {
      const uint32_t nverts = t.vend - t.vbegin;
      const uint32_t ngroups = (nverts + 31) / 32;
      for (uint32_t g = warp; g < ngroups; g += kPrWarps) {
        const uint32_t u = t.vbegin + g * 32 + lane;
        uint32_t ls = 0, deg = 0;
        float c = 0.f;
        if (u < t.vend) {
          const uint64_t e0 = __ldg(a.off + u), e1 = __ldg(a.off + u + 1);
          ls = (uint32_t)(e0 - t.ebegin);
          deg = (uint32_t)(e1 - e0);
          c = __ldg(a.cur + u);
        }
        const unsigned incl = warp_incl_scan<unsigned>(deg);
        const unsigned excl = incl - deg;
        const unsigned total = __shfl_sync(kFull, incl, 31);
        for (unsigned k = 0; k < total; k += 32) {
          const unsigned tt = k + lane;
          const int o = warp_owner(excl, tt);
          const unsigned ols = __shfl_sync(kFull, ls, o);
          const unsigned oex = __shfl_sync(kFull, excl, o);
          const float oc = __shfl_sync(kFull, c, o);
          if (tt < total)
            atomicAdd(a.sum + staged_id<ESZ>(s_e, shift + ols + (tt - oex), a.wshift), (double)oc);
        }
      }
    }
    __syncthreads();
  }
}

__global__ void pr_push_update(PrArgs a) {
  __shared__ double s_red[kPrWarps];
  const double base = (1.0 - a.damping) * a.inv_n + a.damping * ldcg(a.dang + a.it) * a.inv_n;
  double dsum = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    const double s = a.sum[v];
    a.sum[v] = 0.0;
    dsum += finish_vertex(a, v, s, base);
  }
  dsum = block_sum(dsum, s_red);
  if (threadIdx.x == 0 && dsum != 0.0) atomicAdd(a.dang + a.it + 1, dsum);
}

__global__ void pr_init(PrArgs a, float *c0) {
  __shared__ double s_red[kPrWarps];
  double dsum = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    a.rank[v] = (float)a.inv_n;
    const uint32_t od = out_degree(a, v);
    c0[v] = od ? (float)(a.inv_n / (double)od) : 0.f;
    if (!od) dsum += a.inv_n;
    if (a.sum) a.sum[v] = 0.0;
  }
  dsum = block_sum(dsum, s_red);
  if (threadIdx.x == 0 && dsum != 0.0) atomicAdd(a.dang, dsum);
}

// ------------------------------------------- reference semantics (FP64) --
//
// THV_RUN_PR_REFERENCE reproduces the reference engine's own PageRank so its
// values.bin can be compared with the reference comparer's 1e-3 absolute
// tolerance (comparer/compare.cpp:155).  Its constants are floats
// (src/common.cuh:48-49) mixed into double expressions; the same expressions
// here give the same promoted values.
//   pull: r0 = 1/N (src/graph.cuh:239-240); per round every active vertex
//         sums r(u)/outdeg(u) over its in-edges from the previous round's
//         values, then r = (1-a) + a*sum and it stays active while the change
//         exceeds the tolerance (src/pr/pr_kernels.cu:23-55, :449-476);
//   push: r0 = 1-a, delta0 = (1-a)*a/outdeg in float, residual 0
//         (src/graph.cuh:233-237); per round each active u adds delta(u) to
//         residual(w) over its out-edges (pr_kernels.cu:504-681), then every
//         vertex with residual > tol takes it and becomes active, the rest
//         inactive (pr_kernels.cu:846-860, frontier cleared each round at
//         src/pr/pr.cu:1067-1077).
// Rounds run until no vertex is active.  The gather/scatter kernels reuse
// the tiles of the fixed-iteration kernels and skip tiles without an active
// vertex, so converged regions cost one flag read per vertex.  Pull sums are
// warp-segmented (fixed order) with atomics only across the parts of a split
// vertex; push adds with FP64 atomics like the reference.
constexpr float kRefAlpha = 0.85f, kRefTol = 0.001f;

struct PrRefArgs {
  const PrTile *tiles;
  const uint64_t *blk_base;
  const uint64_t *off;
  const uint32_t *outdeg;  // CSC: explicit; CSR: nullptr
  double *val, *acc, *delta;
  uint8_t *act;
  double *split_acc;
  uint32_t *split_done;
  const uint32_t *split_parts;
  uint32_t *tile_ctr;
  unsigned long long *cnt;  // [0] active vertices, [1] their edges
  uint32_t ntiles, nv, wshift, pad;
};

__device__ __forceinline__ uint32_t ref_out_degree(const PrRefArgs &a, uint32_t v) {
  return a.outdeg ? __ldg(a.outdeg + v)
                  : (uint32_t)(__ldg(a.off + v + 1) - __ldg(a.off + v));
}

// Stage edges [t.ebegin, t.eend) of a tile (same layout as stage_tile).
template <int ESZ>
__device__ __forceinline__ uint32_t ref_stage(const PrRefArgs &a, const PrTile &t, uint32_t *s_e) {
  const uintptr_t b = (uintptr_t)__ldg(a.blk_base + t.block);
  const uintptr_t s0 = b + (uintptr_t)t.ebegin * ESZ;
  const uintptr_t s1 = b + (uintptr_t)t.eend * ESZ;
  const uintptr_t a0 = s0 & ~(uintptr_t)15;
  const uint32_t nvec = (uint32_t)((s1 - a0 + 15) / 16);
  uint4 *dst = reinterpret_cast<uint4 *>(s_e);
  for (uint32_t i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = ld_nc_v4(a0 + 16u * i);
  return (uint32_t)((s0 - a0) / ESZ);
}

// Next tile with an active vertex; returns false when the tiles are done.
__device__ __forceinline__ bool ref_next_tile(const PrRefArgs &a, PrTile *t, uint32_t *s_tile) {
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) *s_tile = atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const uint32_t ti = *s_tile;
    if (ti >= a.ntiles) return false;
    *t = a.tiles[ti];
    int any = 0;
    for (uint32_t v = t->vbegin + threadIdx.x; v < t->vend; v += blockDim.x) any |= a.act[v];
    if (__syncthreads_or(any)) return true;
  }
}

template <int ESZ>
__global__ void __launch_bounds__(kPrThreads) pr_ref_pull_kernel(PrRefArgs a) {
  __shared__ __align__(16) uint32_t s_e[kStageEdges * (ESZ / 4) + 16];
  __shared__ double s_acc[kPrWarps][32];
  __shared__ double s_red[kPrWarps];
  __shared__ uint32_t s_tile;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  PrTile t;
  while (ref_next_tile(a, &t, &s_tile)) {
    const uint32_t shift = ref_stage<ESZ>(a, t, s_e);
    __syncthreads();
    if (t.split) {
      const uint32_t cnt = (uint32_t)(t.eend - t.ebegin);
      double part = 0.0;
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
        const uint32_t u = staged_id<ESZ>(s_e, shift + i, a.wshift);
        const uint32_t od = __ldg(a.outdeg + u);
        if (od) part += a.val[u] / (double)od;
      }
      part = block_sum(part, s_red);
      if (threadIdx.x == 0) {
        const uint32_t sv = t.split - 1;
        atomicAdd(a.split_acc + sv, part);
        __threadfence();
        const uint32_t done = atomicAdd(a.split_done + sv, 1u);
        if (done + 1 == __ldg(a.split_parts + sv)) {
          __threadfence();
          const unsigned long long bits =
              atomicExch(reinterpret_cast<unsigned long long *>(a.split_acc + sv), 0ull);
          a.split_done[sv] = 0;
          a.acc[t.vbegin] = __longlong_as_double((long long)bits);
        }
      }
    } else {
      const uint32_t nverts = t.vend - t.vbegin;
      const uint32_t ngroups = (nverts + 31) / 32;
      for (uint32_t g = warp; g < ngroups; g += kPrWarps) {
        const uint32_t v = t.vbegin + g * 32 + lane;
        const bool on = v < t.vend && a.act[v];
        uint32_t ls = 0, deg = 0;
        if (on) {
          const uint64_t e0 = __ldg(a.off + v), e1 = __ldg(a.off + v + 1);
          ls = (uint32_t)(e0 - t.ebegin);
          deg = (uint32_t)(e1 - e0);
        }
        const unsigned incl = warp_incl_scan<unsigned>(deg);
        const unsigned excl = incl - deg;
        const unsigned total = __shfl_sync(kFull, incl, 31);
        s_acc[warp][lane] = 0.0;
        __syncwarp();
        for (unsigned k = 0; k < total; k += 32) {
          const unsigned tt = k + lane;
          const int o = warp_owner(excl, tt);
          const unsigned ols = __shfl_sync(kFull, ls, o);
          const unsigned oex = __shfl_sync(kFull, excl, o);
          double x = 0.0;
          int pos = 32;
          if (tt < total) {
            const uint32_t u = staged_id<ESZ>(s_e, shift + ols + (tt - oex), a.wshift);
            const uint32_t od = __ldg(a.outdeg + u);
            x = od ? a.val[u] / (double)od : 0.0;
            pos = o;
          }
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_up_sync(kFull, x, d);
            const int pp = __shfl_up_sync(kFull, pos, d);
            if (lane >= (unsigned)d && pp == pos) x += y;
          }
          const int nxt = __shfl_down_sync(kFull, pos, 1);
          if ((lane == 31 || nxt != pos) && pos < 32) s_acc[warp][pos] += x;
          __syncwarp();
        }
        if (on) a.acc[v] = s_acc[warp][lane];
        __syncwarp();
      }
    }
  }
}

template <int ESZ>
__global__ void __launch_bounds__(kPrThreads) pr_ref_push_kernel(PrRefArgs a) {
  __shared__ __align__(16) uint32_t s_e[kStageEdges * (ESZ / 4) + 16];
  __shared__ uint32_t s_tile;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  PrTile t;
  while (ref_next_tile(a, &t, &s_tile)) {
    const uint32_t shift = ref_stage<ESZ>(a, t, s_e);
    __syncthreads();
    if (t.split) {
      const double c = a.delta[t.vbegin];
      const uint32_t cnt = (uint32_t)(t.eend - t.ebegin);
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
        atomicAdd(a.acc + staged_id<ESZ>(s_e, shift + i, a.wshift), c);
    } else {
      const uint32_t nverts = t.vend - t.vbegin;
      const uint32_t ngroups = (nverts + 31) / 32;
      for (uint32_t g = warp; g < ngroups; g += kPrWarps) {
        const uint32_t u = t.vbegin + g * 32 + lane;
        uint32_t ls = 0, deg = 0;
        double c = 0.0;
        if (u < t.vend && a.act[u]) {
          const uint64_t e0 = __ldg(a.off + u), e1 = __ldg(a.off + u + 1);
          ls = (uint32_t)(e0 - t.ebegin);
          deg = (uint32_t)(e1 - e0);
          c = a.delta[u];
        }
        const unsigned incl = warp_incl_scan<unsigned>(deg);
        const unsigned excl = incl - deg;
        const unsigned total = __shfl_sync(kFull, incl, 31);
        for (unsigned k = 0; k < total; k += 32) {
          const unsigned tt = k + lane;
          const int o = warp_owner(excl, tt);
          const unsigned ols = __shfl_sync(kFull, ls, o);
          const unsigned oex = __shfl_sync(kFull, excl, o);
          const double oc = __shfl_sync(kFull, c, o);
          if (tt < total) atomicAdd(a.acc + staged_id<ESZ>(s_e, shift + ols + (tt - oex), a.wshift), oc);
        }
      }
    }
  }
}

__device__ __forceinline__ void ref_count(const PrRefArgs &a, unsigned long long nact,
                                          unsigned long long nedge) {
  nact = warp_sum(nact);
  nedge = warp_sum(nedge);
  if (lane_id() == 0 && nact) {
    atomicAdd(a.cnt, nact);
    atomicAdd(a.cnt + 1, nedge);
  }
}

// Edges the next round reads for an active vertex: its in-edges (pull over
// CSC) or its out-edges (push over CSR), both given by the offsets.
__device__ __forceinline__ uint32_t ref_edges(const PrRefArgs &a, uint32_t v) {
  return (uint32_t)(__ldg(a.off + v + 1) - __ldg(a.off + v));
}

__global__ void pr_ref_init(PrRefArgs a, int push) {
  unsigned long long nact = 0, nedge = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    a.act[v] = 1;
    a.acc[v] = 0.0;
    if (push) {
      a.val[v] = (double)(1.0f - kRefAlpha);
      a.delta[v] = (double)((1.0f - kRefAlpha) * kRefAlpha / (float)ref_out_degree(a, v));
    } else {
      a.val[v] = 1.0 / (double)a.nv;
    }
    nact++;
    nedge += ref_edges(a, v);
  }
  ref_count(a, nact, nedge);
}

__global__ void pr_ref_pull_update(PrRefArgs a) {
  unsigned long long nact = 0, nedge = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    if (!a.act[v]) continue;
    const double t = (1 - kRefAlpha) + kRefAlpha * a.acc[v];
    const double old = a.val[v];
    const double diff = t > old ? t - old : old - t;
    a.val[v] = t;
    const bool on = diff > kRefTol;
    a.act[v] = on;
    if (on) {
      nact++;
      nedge += ref_edges(a, v);
    }
  }
  ref_count(a, nact, nedge);
}

__global__ void pr_ref_push_update(PrRefArgs a) {
  unsigned long long nact = 0, nedge = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    const double r = a.acc[v];
    const bool on = r > kRefTol;
    if (on) {
      a.val[v] += r;
      a.delta[v] = r * kRefAlpha / (double)ref_out_degree(a, v);
      a.acc[v] = 0.0;
      nact++;
      nedge += ref_edges(a, v);
    }
    a.act[v] = on;
  }
  ref_count(a, nact, nedge);
}

// ------------------------------------------------------------------ host --

void pagerank_free(thv_graph *g) {
  PrState *p = g->ps;
  if (!p) return;
  dev_free(p->d_c[0]);
  dev_free(p->d_c[1]);
  dev_free(p->d_rank);
  dev_free(p->d_sum);
  dev_free(p->d_split_acc);
  dev_free(p->d_split_done);
  dev_free(p->d_dang);
  dev_free(p->d_tile_ctr);
  dev_free(p->d_val);
  dev_free(p->d_acc);
  dev_free(p->d_delta);
  dev_free(p->d_act);
  dev_free(p->d_cnt);
  pinned_free(p->h_cnt);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  delete p;
  g->ps = nullptr;
}

static thv_status ensure_pr_state(thv_graph *g, bool push, uint32_t iters, bool ref) {
  PrState *&p = g->ps;
  const size_t nsplit = std::max<size_t>(1, g->plan.split_parts.size());
  if (p && p->push == push && p->ref == ref && (ref || p->cap_iters >= iters) && p->nsplit == nsplit)
    return THV_OK;
  pagerank_free(g);
  p = new PrState();
  p->nv = g->nv;
  p->push = push;
  p->ref = ref;
  p->nsplit = nsplit;
  if (ref) {
    THV_TRY(dev_alloc((void **)&p->d_val, g->nv * 8 + 64, "pr values"));
    THV_TRY(dev_alloc((void **)&p->d_acc, g->nv * 8 + 64, "pr sums"));
    if (push) THV_TRY(dev_alloc((void **)&p->d_delta, g->nv * 8 + 64, "pr deltas"));
    THV_TRY(dev_alloc((void **)&p->d_act, g->nv + 64, "pr active flags"));
    THV_TRY(dev_alloc((void **)&p->d_cnt, 16, "pr round counters"));
    THV_TRY(pinned_alloc((void **)&p->h_cnt, 16, "pr round counters"));
    THV_TRY(dev_alloc((void **)&p->d_split_acc, nsplit * 8, "pr split sums"));
    THV_TRY(dev_alloc((void **)&p->d_split_done, nsplit * 4, "pr split counters"));
    THV_TRY(dev_alloc((void **)&p->d_tile_ctr, 4, "pr tile counter"));
    THV_CUDA(cudaEventCreate(&p->ev0));
    THV_CUDA(cudaEventCreate(&p->ev1));
    return THV_OK;
  }
  p->cap_iters = std::max<uint32_t>(iters, 32);
  THV_TRY(dev_alloc((void **)&p->d_c[0], g->nv * 4 + 64, "pr contributions"));
  THV_TRY(dev_alloc((void **)&p->d_c[1], g->nv * 4 + 64, "pr contributions"));
  THV_TRY(dev_alloc((void **)&p->d_rank, g->nv * 4 + 64, "pr ranks"));
  if (push) THV_TRY(dev_alloc((void **)&p->d_sum, g->nv * 8 + 64, "pr sums"));
  THV_TRY(dev_alloc((void **)&p->d_split_acc, nsplit * 8, "pr split sums"));
  THV_TRY(dev_alloc((void **)&p->d_split_done, nsplit * 4, "pr split counters"));
  THV_TRY(dev_alloc((void **)&p->d_dang, (p->cap_iters + 1) * 8, "pr dangling"));
  THV_TRY(dev_alloc((void **)&p->d_tile_ctr, p->cap_iters * 4, "pr tile counters"));
  THV_CUDA(cudaEventCreate(&p->ev0));
  THV_CUDA(cudaEventCreate(&p->ev1));
  return THV_OK;
}

template <int ESZ>
static thv_status pr_iterate(thv_graph *g, PrArgs &a, bool push, uint32_t iters,
                             cudaStream_t st, uint32_t &launches) {
  PrState *p = g->ps;
  int bpsm = 0;
  if (push)
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, pr_push_kernel<ESZ>, kPrThreads, 0));
  else
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, pr_pull_kernel<ESZ>, kPrThreads, 0));
  const int grid = std::max(1, bpsm) * g->num_sms;
  const int ugrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + kPrThreads - 1) / kPrThreads)));
  for (uint32_t it = 0; it < iters; it++) {
    a.it = it;
    a.cur = p->d_c[it & 1];
    a.nxt = p->d_c[(it + 1) & 1];
    if (push) {
      pr_push_kernel<ESZ><<<grid, kPrThreads, 0, st>>>(a);
      pr_push_update<<<ugrid, kPrThreads, 0, st>>>(a);
      launches += 2;
    } else {
      pr_pull_kernel<ESZ><<<grid, kPrThreads, 0, st>>>(a);
      launches += 1;
    }
    THV_CUDA(cudaGetLastError());
  }
  return THV_OK;
}

// Reference semantics: one gather/scatter launch and one update launch per
// round; the host reads the round's active count (16 bytes) to stop.
static thv_status run_pagerank_ref(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                                   cudaStream_t st, thv_stats *stats) {
  const bool push = algo == THV_ALGO_PR_PUSH;
  const uint32_t max_rounds = o && o->pr_iters ? o->pr_iters : 100000u;
  THV_TRY(ensure_plan(g));
  THV_TRY(build_tiles(g));
  THV_TRY(ensure_pr_state(g, push, 0, true));
  PrState *p = g->ps;
  PrRefArgs a{};
  a.tiles = g->plan.d_tiles;
  a.blk_base = g->plan.d_base;
  a.off = g->d_off;
  a.outdeg = g->fmt == THV_FMT_CSC ? g->d_outdeg : nullptr;
  a.val = p->d_val;
  a.acc = p->d_acc;
  a.delta = p->d_delta;
  a.act = p->d_act;
  a.split_acc = p->d_split_acc;
  a.split_done = p->d_split_done;
  a.split_parts = g->plan.d_split_parts;
  a.tile_ctr = p->d_tile_ctr;
  a.cnt = p->d_cnt;
  a.ntiles = (uint32_t)g->plan.tiles.size();
  a.nv = (uint32_t)g->nv;
  a.wshift = g->wshift;
  int bpsm = 0;
  if (push)
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, g->esz == 8 ? pr_ref_push_kernel<8> : pr_ref_push_kernel<4>, kPrThreads, 0));
  else
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, g->esz == 8 ? pr_ref_pull_kernel<8> : pr_ref_pull_kernel<4>, kPrThreads, 0));
  const int grid = std::max(1, bpsm) * g->num_sms;
  const int ugrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + kPrThreads - 1) / kPrThreads)));
  const size_t nsplit = std::max<size_t>(1, g->plan.split_parts.size());
  uint32_t launches = 0, rounds = 0;
  uint64_t edges = 0;
  THV_CUDA(cudaEventRecord(p->ev0, st));
  THV_CUDA(cudaMemsetAsync(p->d_split_acc, 0, nsplit * 8, st));
  THV_CUDA(cudaMemsetAsync(p->d_split_done, 0, nsplit * 4, st));
  THV_CUDA(cudaMemsetAsync(p->d_cnt, 0, 16, st));
  pr_ref_init<<<ugrid, kPrThreads, 0, st>>>(a, push ? 1 : 0);
  THV_CUDA(cudaGetLastError());
  launches++;
  THV_CUDA(cudaMemcpyAsync(p->h_cnt, p->d_cnt, 16, cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaStreamSynchronize(st));
  while (p->h_cnt[0]) {
    if (rounds == max_rounds) return fail(THV_ETIMEOUT, "PageRank did not converge in %u rounds", max_rounds);
    edges += p->h_cnt[1];
    THV_CUDA(cudaMemsetAsync(p->d_tile_ctr, 0, 4, st));
    THV_CUDA(cudaMemsetAsync(p->d_cnt, 0, 16, st));
    if (push) {
      if (g->esz == 8) pr_ref_push_kernel<8><<<grid, kPrThreads, 0, st>>>(a);
      else pr_ref_push_kernel<4><<<grid, kPrThreads, 0, st>>>(a);
      pr_ref_push_update<<<ugrid, kPrThreads, 0, st>>>(a);
    } else {
      if (g->esz == 8) pr_ref_pull_kernel<8><<<grid, kPrThreads, 0, st>>>(a);
      else pr_ref_pull_kernel<4><<<grid, kPrThreads, 0, st>>>(a);
      pr_ref_pull_update<<<ugrid, kPrThreads, 0, st>>>(a);
    }
    THV_CUDA(cudaGetLastError());
    launches += 2;
    THV_CUDA(cudaMemcpyAsync(p->h_cnt, p->d_cnt, 16, cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaStreamSynchronize(st));
    rounds++;
  }
  THV_CUDA(cudaEventRecord(p->ev1, st));
  THV_CUDA(cudaStreamSynchronize(st));
  g->last_algo = algo;
  if (stats) {
    float ms_ = 0.f;
    cudaEventElapsedTime(&ms_, p->ev0, p->ev1);
    stats->device_ms = ms_;
    stats->iterations = rounds;
    stats->edges_expanded = edges;
    stats->kernel_launches = launches;
  }
  return THV_OK;
}

thv_status run_pagerank(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                        cudaStream_t st, thv_stats *stats) {
  const bool push = algo == THV_ALGO_PR_PUSH;
  if (push && g->fmt == THV_FMT_CSC)
    return fail(THV_EINVAL, "push PageRank needs out-edges (CSR), got CSC");
  if (!push && g->fmt != THV_FMT_CSC)
    return fail(THV_EINVAL, "pull PageRank needs in-edges (CSC)");
  if (g->nv == 0) return fail(THV_EINVAL, "empty graph");
  if (o && (o->flags & THV_RUN_PR_REFERENCE)) return run_pagerank_ref(g, algo, o, st, stats);
  const uint32_t iters = o && o->pr_iters ? o->pr_iters : 20u;
  const double damping = o && o->pr_damping > 0 ? o->pr_damping : 0.85;
  THV_TRY(ensure_plan(g));
  THV_TRY(build_tiles(g));
  THV_TRY(ensure_pr_state(g, push, iters, false));
  PrState *p = g->ps;
  p->iters = iters;

  PrArgs a{};
  a.tiles = g->plan.d_tiles;
  a.blk_base = g->plan.d_base;
  a.off = g->d_off;
  a.outdeg = g->fmt == THV_FMT_CSC ? g->d_outdeg : nullptr;
  a.rank = p->d_rank;
  a.sum = p->d_sum;
  a.split_acc = p->d_split_acc;
  a.split_done = p->d_split_done;
  a.split_parts = g->plan.d_split_parts;
  a.dang = p->d_dang;
  a.tile_ctr = p->d_tile_ctr;
  a.ntiles = (uint32_t)g->plan.tiles.size();
  a.nv = (uint32_t)g->nv;
  a.damping = damping;
  a.inv_n = 1.0 / (double)g->nv;
  a.wshift = g->wshift;

  uint32_t launches = 0;
  THV_CUDA(cudaEventRecord(p->ev0, st));
  THV_CUDA(cudaMemsetAsync(p->d_dang, 0, (iters + 1) * 8, st));
  THV_CUDA(cudaMemsetAsync(p->d_tile_ctr, 0, iters * 4, st));
  const size_t nsplit = std::max<size_t>(1, g->plan.split_parts.size());
  THV_CUDA(cudaMemsetAsync(p->d_split_acc, 0, nsplit * 8, st));
  THV_CUDA(cudaMemsetAsync(p->d_split_done, 0, nsplit * 4, st));
  const int ugrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + kPrThreads - 1) / kPrThreads)));
  pr_init<<<ugrid, kPrThreads, 0, st>>>(a, p->d_c[0]);
  THV_CUDA(cudaGetLastError());
  launches++;
  thv_status s = g->esz == 8 ? pr_iterate<8>(g, a, push, iters, st, launches)
                             : pr_iterate<4>(g, a, push, iters, st, launches);
  if (s != THV_OK) return s;
  THV_CUDA(cudaEventRecord(p->ev1, st));
  THV_CUDA(cudaStreamSynchronize(st));
  g->last_algo = algo;
  if (stats) {
    float ms_ = 0.f;
    cudaEventElapsedTime(&ms_, p->ev0, p->ev1);
    stats->device_ms = ms_;
    stats->iterations = iters;
    stats->edges_expanded = g->ne * iters;
    stats->hbm_edge_bytes = g->plan.tiles_hbm_bytes * iters;
    stats->link_edge_bytes = g->plan.tiles_link_bytes * iters;
    stats->kernel_launches = launches;
  }
  return THV_OK;
}

thv_status pagerank_values(thv_graph *g, double *out, cudaStream_t st) {
  if (!g->ps) return fail(THV_EINVAL, "no PageRank values");
  if (g->ps->ref) {
    THV_CUDA(cudaMemcpyAsync(out, g->ps->d_val, g->nv * 8, cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaStreamSynchronize(st));
    return THV_OK;
  }
  std::vector<float> tmp(g->nv);
  THV_CUDA(cudaMemcpyAsync(tmp.data(), g->ps->d_rank, g->nv * 4, cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaStreamSynchronize(st));
  for (uint64_t i = 0; i < g->nv; i++) out[i] = (double)tmp[i];
  return THV_OK;
}

}  // namespace thv
