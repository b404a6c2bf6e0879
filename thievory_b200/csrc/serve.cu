// Serving: continuous batching of BFS / SSSP queries over one resident graph.
//
// No counterpart in the reference (one query per process, src/main.cu:152).
// Up to 64 queries occupy the slots of a single traversal state
//   val[v][slot]   u32, value + 1 in the single-source encoding (n+1 unset)
//   front[v]       u64 mask of slots for which v is pending
// driven by the frontier machinery of the single-source engine (pending
// bitmap, ballot compaction into small-vertex groups and high-degree chunks,
// zero-copy addressing), with per-slot near/far thresholds so that queries
// admitted at different times coexist.  BFS slots relax with unit weights
// (distance + 1 == level + 1, window 1: exactly level-synchronous); SSSP
// slots use the edge weights with window 64: wide enough that many slots
// expand the same vertex in the same iteration and share its edge read.
//
// The persistent kernel returns to the host when any slot's query has no
// pending vertex left, or after a bounded number of iterations when
// requests are waiting.  The host dispatcher thread then writes finished
// slots' results (one column of val) into the caller's buffers, resets the
// column, admits waiting requests into free slots (seeding their sources)
// and relaunches: a request that arrives while others run joins at the next
// launch boundary and shares every later edge read with them.
//
// The default mode runs the same admission on the batched kernels instead
// (batch.cu, live groups): one group per algorithm with 64-bit source
// masks (BFS levels in bytes, SSSP distances in 64-wide rows), each launch
// running one iteration or a few, finished sources retiring and waiting
// queries joining free mask bits between launches; the BFS and SSSP groups
// take turns on the device.  An idle server runs a lone query on the
// single-source kernel, which is faster for one query than a group.
#include <algorithm>
#include <chrono>
#include <cstddef>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

constexpr int kSvThreads = 512;
constexpr uint32_t kSvMaxSlots = 64;
constexpr uint32_t kSvDeltaSssp = 256;  // shared-read sweet spot (batched sweep)

struct SvCtrl {
  GridBar bar;
  unsigned err, iters;
  unsigned long long cnt_small[3], cnt_big[3], wc[3];
  unsigned long long taken_or[3], alive_or[3];
  unsigned thr[kSvMaxSlots], step[kSvMaxSlots];
  unsigned long long done_mask;
  unsigned long long edges, hbm_bytes, link_bytes, pairs;
};

struct SvArgs {
  const uint64_t *off;
  const uint32_t *blk_vb;
  const uint64_t *blk_base;
  uint64_t host_base;
  ListCache lc;
  unsigned long long *blk_access;  // tracked plans: adjacency bytes read per block
  uint32_t *val;  // [nv][W]
  unsigned long long *front;
  uint32_t *bm;
  WorkItem *qs, *qb;
  unsigned long long *qsm, *qbm;
  unsigned long long cap_s, cap_b;
  SvCtrl *ctrl;
  unsigned long long active, unit;
  unsigned long long timeout_ns;
  uint32_t nblk, nv, ngroups, W;
  uint32_t max_iters, small_deg, chunk;
  uint32_t wshift, wbase;  // 4-byte edges: see edge_dst / edge_wt
  uint32_t pad;
};

__device__ __forceinline__ void sv_edge(const SvArgs &a, uint32_t u, uint32_t w, uint32_t wt,
                                        unsigned long long f) {
  const uint32_t *du = a.val + (size_t)u * a.W;
  uint32_t *dw = a.val + (size_t)w * a.W;
  unsigned long long improved = 0;
  while (f) {
    const int s = __ffsll((long long)f) - 1;
    f &= f - 1;
    const unsigned long long cand =
        (unsigned long long)ldcg(du + s) + (((a.unit >> s) & 1ull) ? 1u : wt);
    if (cand < ldcg(dw + s)) {
      const uint32_t old = atomicMin(dw + s, (uint32_t)cand);
      if (cand < old) improved |= 1ull << s;
    }
  }
  if (improved) {
    atomicOr(a.front + w, improved);
    const uint32_t m = 1u << (w & 31u);
    uint32_t *bp = a.bm + (w >> 5);
    if (!(ldcg(bp) & m)) atomicOr(bp, m);
  }
}

// Lane-per-slot relaxation of one work item (dense masks): edges loaded 32
// at a time, each relaxed for all slots of the mask at once with lanes =
// slots, so val[w][.] is read as coalesced lines; four rows in flight.
template <int ESZ>
__device__ __forceinline__ void sv_item_rows(const SvArgs &a, uint32_t u, uintptr_t eaddr,
                                             uint32_t cnt, unsigned long long f) {
  const unsigned lane = lane_id();
  const bool lo = (f >> lane) & 1ull, hi = (f >> (lane + 32)) & 1ull;
  const uint32_t one0 = (uint32_t)((a.unit >> lane) & 1ull);
  const uint32_t one1 = (uint32_t)((a.unit >> (lane + 32)) & 1ull);
  const uint32_t *du = a.val + (size_t)u * a.W;
  const uint32_t d0 = lo ? ldcg(du + lane) : 0u, d1 = hi ? ldcg(du + 32 + lane) : 0u;
  for (uint32_t base = 0; base < cnt; base += 32) {
    const uint32_t k = base + lane;
    uint32_t ex = 0, ey = 1;
    if (k < cnt) {
      if (ESZ == 4) {
        const uint32_t r = ld_nc_u32(eaddr + (uintptr_t)k * 4u);
        ex = edge_dst(r, a.wshift);
        ey = edge_wt(r, a.wshift, a.wbase);
      } else {
        const uint2 e = ld_nc_u2(eaddr + (uintptr_t)k * 8u);
        ex = e.x;
        ey = e.y;
      }
    }
    const uint32_t m = min(32u, cnt - base);
    for (uint32_t j = 0; j < m; j += 4) {
      uint32_t w[4], wt[4], c0[4], c1[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        w[q] = __shfl_sync(kFull, ex, (j + q) & 31);
        wt[q] = __shfl_sync(kFull, ey, (j + q) & 31);
        const bool ok = j + q < m;
        const uint32_t *dw = a.val + (size_t)w[q] * a.W;
        c0[q] = ok && lo ? ldcg(dw + lane) : 0u;
        c1[q] = ok && hi ? ldcg(dw + 32 + lane) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (j + q >= m) break;
        uint32_t *dw = a.val + (size_t)w[q] * a.W;
        const unsigned long long cd0 = (unsigned long long)d0 + (one0 ? 1u : wt[q]);
        const unsigned long long cd1 = (unsigned long long)d1 + (one1 ? 1u : wt[q]);
        const bool i0 = lo && cd0 < c0[q] && cd0 < atomicMin(dw + lane, (uint32_t)cd0);
        const bool i1 = hi && cd1 < c1[q] && cd1 < atomicMin(dw + 32 + lane, (uint32_t)cd1);
        const unsigned b0 = __ballot_sync(kFull, i0), b1 = __ballot_sync(kFull, i1);
        if ((b0 | b1) && lane == 0) {
          atomicOr(a.front + w[q], (unsigned long long)b0 | ((unsigned long long)b1 << 32));
          const uint32_t mb = 1u << (w[q] & 31u);
          uint32_t *bp = a.bm + (w[q] >> 5);
          if (!(ldcg(bp) & mb)) atomicOr(bp, mb);
        }
      }
    }
  }
}

constexpr int kSvSparseMask = 4;

template <int ESZ>
__device__ __forceinline__ void sv_chunk(const SvArgs &a, const WorkItem &it, unsigned long long f) {
  if (__popcll(f) > kSvSparseMask) {
    sv_item_rows<ESZ>(a, it.v, it.eaddr, it.cnt, f);
    return;
  }
  constexpr int PER = 16 / ESZ;
  const unsigned lane = lane_id();
  const uintptr_t start = it.eaddr;
  const uintptr_t end = start + (uintptr_t)it.cnt * ESZ;
  for (uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane; p < end; p += 512u) {
    const uint4 q = ld_nc_v4(p);
    const uint32_t e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const uintptr_t ea = p + (uintptr_t)ESZ * j;
      if (ea >= start && ea < end)
        sv_edge(a, it.v, ESZ == 4 ? edge_dst(e[j], a.wshift) : e[2 * j],
                ESZ == 4 ? edge_wt(e[j], a.wshift, a.wbase) : e[2 * j + 1], f);
    }
  }
}

template <int ESZ>
__device__ __forceinline__ void sv_group(const SvArgs &a, unsigned long long first,
                                         unsigned long long n_small) {
  const unsigned lane = lane_id();
  const unsigned long long idx = first + lane;
  WorkItem it{0, 0, 0};
  unsigned long long f = 0;
  if (idx < n_small) {
    it = a.qs[idx];
    f = a.qsm[idx];
  }
  unsigned dense = __ballot_sync(kFull, __popcll(f) > kSvSparseMask);
  while (dense) {
    const int i = __ffs(dense) - 1;
    dense &= dense - 1;
    sv_item_rows<ESZ>(a, __shfl_sync(kFull, it.v, i), (uintptr_t)shfl64(it.eaddr, i),
                      __shfl_sync(kFull, it.cnt, i), shfl64(f, i));
  }
  if (__popcll(f) > kSvSparseMask) {
    it.cnt = 0;
    f = 0;
  }
  const unsigned incl = warp_incl_scan<unsigned>(it.cnt);
  const unsigned excl = incl - it.cnt;
  const unsigned total = __shfl_sync(kFull, incl, 31);
  for (unsigned k = 0; k < total; k += 32) {
    const unsigned t = k + lane;
    const int o = warp_owner(excl, t);
    const unsigned long long ea = shfl64(it.eaddr, o);
    const unsigned oex = __shfl_sync(kFull, excl, o);
    const unsigned ou = __shfl_sync(kFull, it.v, o);
    const unsigned long long of = shfl64(f, o);
    if (t < total) {
      const uintptr_t addr = (uintptr_t)ea + (uintptr_t)(t - oex) * ESZ;
      if (ESZ == 4) {
        const uint32_t r = ld_nc_u32(addr);
        sv_edge(a, ou, edge_dst(r, a.wshift), edge_wt(r, a.wshift, a.wbase), of);
      } else {
        const uint2 e = ld_nc_u2(addr);
        sv_edge(a, ou, e.x, e.y, of);
      }
    }
  }
}

template <int ESZ>
__global__ void __launch_bounds__(kSvThreads) sv_kernel(SvArgs a) {
  extern __shared__ uint32_t s_dyn[];
  __shared__ uint32_t s_thr[kSvMaxSlots], s_step[kSvMaxSlots];
  uint32_t *s_vb = s_dyn;
  const bool smem_tab = a.nblk <= kSmemBlocks;
  if (smem_tab)
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];
  for (uint32_t s = threadIdx.x; s < kSvMaxSlots; s += blockDim.x) {
    s_thr[s] = ldcg(&a.ctrl->thr[s]);
    s_step[s] = ldcg(&a.ctrl->step[s]);
  }
  __syncthreads();
  const uint32_t *vb = smem_tab ? s_vb : a.blk_vb;
  SvCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  unsigned iter = 0;
  unsigned long long done = 0;
  for (; iter < a.max_iters; ++iter) {
    const unsigned slot = iter % 3, nslot = (iter + 1) % 3;
    if (leader) {
      c->cnt_small[nslot] = 0;
      c->cnt_big[nslot] = 0;
      c->wc[nslot] = 0;
      c->taken_or[nslot] = 0;
      c->alive_or[nslot] = 0;
    }
    // ---------------------------------------------------------- compaction
    unsigned long long my_taken = 0, my_alive = 0, my_edges = 0, my_hbm = 0, my_link = 0,
                       my_pairs = 0;
    for (unsigned g = gwarp; g < a.ngroups; g += nwarps) {
      const unsigned wbase = g * 32u;
      const uint32_t word = ldcg(a.bm + wbase + lane);
      unsigned nz = __ballot_sync(kFull, word != 0);
      while (nz) {
        const int j = __ffs(nz) - 1;
        nz &= nz - 1;
        const uint32_t wd = __shfl_sync(kFull, word, j);
        const uint32_t v = (wbase + j) * 32u + lane;
        unsigned long long take = 0, keep = 0;
        if ((wd >> lane) & 1u) {
          const unsigned long long f = ldcg(a.front + v);
          const uint32_t *dv = a.val + (size_t)v * a.W;
          unsigned long long r = f;
          while (r) {
            const int s = __ffsll((long long)r) - 1;
            r &= r - 1;
            if (ldcg(dv + s) < s_thr[s]) take |= 1ull << s;
          }
          keep = f & ~take;
          a.front[v] = keep;
          my_alive |= f;
          my_taken |= take;
        }
        const unsigned km = __ballot_sync(kFull, keep != 0);
        if (lane == 0) a.bm[wbase + j] = km;
        uint32_t deg = 0;
        unsigned long long eaddr = 0;
        if (take) {
          const uint64_t s0 = __ldg(a.off + v), e0 = __ldg(a.off + v + 1);
          deg = (uint32_t)(e0 - s0);
          bool host;
          const uint32_t bi = find_block(vb, a.nblk, v);
          eaddr = list_addr(a.lc, __ldg(a.blk_base + bi), a.host_base, v, s0, deg, ESZ, &host);
          if (a.blk_access) atomicAdd(a.blk_access + bi, (unsigned long long)deg * ESZ);
          my_edges += deg;
          my_pairs += __popcll(take);
          if (host) my_link += (unsigned long long)deg * ESZ;
          else my_hbm += (unsigned long long)deg * ESZ;
        }
        const bool small = take && deg > 0 && deg < a.small_deg;
        const bool big = take && deg >= a.small_deg;
        const unsigned sm = __ballot_sync(kFull, small);
        if (sm) {
          const int ldr = __ffs(sm) - 1;
          unsigned long long base = 0;
          if (lane == (unsigned)ldr)
            base = atomicAdd(&c->cnt_small[slot], (unsigned long long)__popc(sm));
          base = shfl64(base, ldr);
          const unsigned long long pos = base + __popc(sm & lanemask_lt());
          if (small) {
            if (pos < a.cap_s) {
              a.qs[pos] = WorkItem{eaddr, v, deg};
              a.qsm[pos] = take;
            } else {
              atomicCAS(&c->err, 0u, kDevErrQueue);
            }
          }
        }
        if (__any_sync(kFull, big)) {
          const unsigned nch = big ? (deg + a.chunk - 1) / a.chunk : 0u;
          const unsigned inc = warp_incl_scan<unsigned>(nch);
          const unsigned tot = __shfl_sync(kFull, inc, 31);
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(&c->cnt_big[slot], (unsigned long long)tot);
          base = shfl64(base, 0);
          if (big) {
            unsigned long long pos = base + inc - nch;
            for (unsigned k = 0; k < nch; k++, pos++) {
              const uint32_t lo = k * a.chunk;
              if (pos < a.cap_b) {
                a.qb[pos] = WorkItem{eaddr + (unsigned long long)lo * ESZ, v, min(a.chunk, deg - lo)};
                a.qbm[pos] = take;
              } else {
                atomicCAS(&c->err, 0u, kDevErrQueue);
              }
            }
          }
        }
      }
    }
    my_taken = warp_or(my_taken);
    my_alive = warp_or(my_alive);
    my_edges = warp_sum(my_edges);
    my_hbm = warp_sum(my_hbm);
    my_link = warp_sum(my_link);
    my_pairs = warp_sum(my_pairs);
    if (lane == 0) {
      if (my_taken) atomicOr(&c->taken_or[slot], my_taken);
      if (my_alive) atomicOr(&c->alive_or[slot], my_alive);
      if (my_pairs) {
        atomicAdd(&c->edges, my_edges);
        atomicAdd(&c->hbm_bytes, my_hbm);
        atomicAdd(&c->link_bytes, my_link);
        atomicAdd(&c->pairs, my_pairs);
      }
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
    const unsigned long long taken = ldcg(&c->taken_or[slot]);
    const unsigned long long alive = ldcg(&c->alive_or[slot]);
    done = a.active & ~alive;
    const unsigned long long ns = ldcg(&c->cnt_small[slot]);
    const unsigned long long nb = ldcg(&c->cnt_big[slot]);
    // ----------------------------------------------------------- expansion
    const unsigned long long ntask = nb + (ns + 31) / 32;
    for (unsigned long long t = gwarp; t < ntask;) {
      if (t < nb) sv_chunk<ESZ>(a, a.qb[t], a.qbm[t]);
      else sv_group<ESZ>(a, (t - nb) * 32ull, ns);
      unsigned long long nt = 0;
      if (lane == 0) nt = nwarps + atomicAdd(&c->wc[slot], 1ull);
      t = shfl64(nt, 0);
    }
    // per-slot windows (one thread per slot; every block computes the same
    // values from the same masks): a slot that expanded something moves by
    // its base width, a pending slot with nothing in its window doubles its
    // step, so a gap in its distances closes in a few iterations
    if (threadIdx.x < kSvMaxSlots && ((a.active >> threadIdx.x) & 1ull)) {
      const uint32_t s = threadIdx.x;
      const uint32_t base = ((a.unit >> s) & 1ull) ? 1u : kSvDeltaSssp;
      uint32_t st = s_step[s];
      if ((taken >> s) & 1ull) st = base;
      else if ((alive >> s) & 1ull) st = min(st * 2u, 1u << 30);
      s_step[s] = st;
      s_thr[s] = (uint32_t)min((unsigned long long)s_thr[s] + st, 0xFFFFFFFFull);
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
    if (done) {
      ++iter;
      break;
    }
  }
  if (leader) {
    c->iters = iter;
    c->done_mask = done;
    for (uint32_t s = 0; s < kSvMaxSlots; s++) {
      c->thr[s] = s_thr[s];
      c->step[s] = s_step[s];
    }
  }
}

__global__ void sv_reset(SvArgs a, uint32_t nw_alloc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t inf = a.nv + 1u;
  for (uint64_t i = tid; i < (uint64_t)a.nv * a.W; i += stride) a.val[i] = inf;
  for (uint64_t v = tid; v < a.nv; v += stride) a.front[v] = 0;
  for (uint64_t w = tid; w < nw_alloc; w += stride) a.bm[w] = 0;
  if (tid == 0) memset(a.ctrl, 0, sizeof(SvCtrl));
}

struct SvSeed {
  uint32_t slot, source, thr, step;
};

__global__ void sv_seed(SvArgs a, const SvSeed *seeds, uint32_t n) {
  const uint32_t i = threadIdx.x;
  if (i >= n) return;
  const SvSeed sd = seeds[i];
  a.val[(size_t)sd.source * a.W + sd.slot] = 1;
  atomicOr(a.front + sd.source, 1ull << sd.slot);
  atomicOr(a.bm + (sd.source >> 5), 1u << (sd.source & 31u));
  a.ctrl->thr[sd.slot] = sd.thr;
  a.ctrl->step[sd.slot] = sd.step;
}

__device__ __forceinline__ unsigned long long sv_hash(uint32_t v, uint32_t val) {
  unsigned long long x = ((unsigned long long)v << 32) | val;
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Column `slot` -> out (may be null), checksum, and reset for reuse.
__global__ void sv_extract(SvArgs a, uint32_t slot, uint32_t *out, unsigned long long *sum) {
  __shared__ unsigned long long s_red[32];
  const uint32_t inf = a.nv + 1u;
  unsigned long long h = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < a.nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t *p = a.val + v * a.W + slot;
    const uint32_t x = *p;
    *p = inf;
    if (out) out[v] = x;
    h += sv_hash((uint32_t)v, x);
  }
  h = warp_sum(h);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = h;
  __syncthreads();
  if (threadIdx.x < 32) {
    h = threadIdx.x < (blockDim.x >> 5) ? s_red[threadIdx.x] : 0ull;
    h = warp_sum(h);
    if (threadIdx.x == 0) atomicAdd(sum, h);
  }
}

}  // namespace thv

// ================================================================== server

using namespace thv;

namespace {

struct Query {
  thv_algo algo;
  uint32_t source;
  uint32_t *out;
  double t_submit = 0, t_start = 0, t_done = 0;
  uint32_t slot = 0, iter_start = 0, iterations = 0;
  uint64_t checksum = 0;
  thv_status status = THV_OK;
  bool done = false;
  uint32_t mode = 0;  // 0 slot, 1 batched group, 2 single-source run
  bool joined = false;  // admitted into a batched group that was already running
};

// Batched-group mode: device bytes per vertex of the batch state (masks,
// 64 distance or level columns, 64-column output staging, queues).
constexpr uint64_t kGroupBytesPerVertex = 600;
// Smallest group worth a batched launch, per algorithm: below it the waiting
// queries run one after another on the single-source kernel.  RMAT-26, 47%
// HBM: a batched group of k BFS sources beats k single runs from k = 4
// (1.16x; 3: 0.91x), of k SSSP sources from k = 6 (1.17x; 4: 0.90x).
constexpr uint32_t kGroupMinBfs = 4, kGroupMinSssp = 6;
constexpr uint32_t kGroupMax = 64;
// Iterations a running group admits arrivals.  RMAT-26 edge factor 48, 256
// queries (80% BFS), Poisson arrivals at 32x the single-run capacity:
// admitting for a group's whole life 61.8 q/s (p99 3.3 s), for its first 2
// iterations 98.2 q/s (p99 1.9 s), only at its start 85.1 q/s; at 4x the
// capacity p50 2.3 s / 0.93 s / 0.91 s.  Sources that start more than a
// level or two apart share few edge reads.
constexpr uint32_t kJoinWindow = 2;

}  // namespace

struct thv_server {
  thv_graph *g = nullptr;
  uint32_t W = 0, queue_cap = 0, batch_iters = 4;
  bool batching = true;    // batched groups + lone runs (false: slots)
  uint32_t group_min = 0;  // explicit group threshold; 0 = per algorithm
  uint32_t replan_every = 0;        // queries between access re-placements
  uint32_t join_window = 0;         // iterations a running group admits arrivals; 0 = always
  uint64_t done_since_replan = 0;
  uint64_t timeout_ns = 0;
  // device state
  uint32_t *d_val = nullptr, *d_bm = nullptr, *d_out = nullptr;
  unsigned long long *d_front = nullptr, *d_qsm = nullptr, *d_qbm = nullptr, *d_sum = nullptr;
  WorkItem *d_qs = nullptr, *d_qb = nullptr;
  uint64_t cap_s = 0, cap_b = 0;
  SvCtrl *d_ctrl = nullptr, *h_ctrl = nullptr;
  SvSeed *d_seeds = nullptr, *h_seeds = nullptr;
  unsigned long long *h_sum = nullptr;
  uint32_t ngroups = 0;
  cudaStream_t st = nullptr;
  // host state
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> waiting;
  std::map<uint64_t, Query> queries;
  uint64_t next_ticket = 1;
  uint64_t slot_ticket[kSvMaxSlots] = {};
  unsigned long long active = 0, unit = 0;
  uint64_t total_iters = 0;
  bool stopping = false;
  thv_status fatal = THV_OK;
  std::string fatal_msg;
  std::thread worker;
  // batching: up to kLiveGroups live groups per algorithm (BFS, SSSP), and
  // the ticket and start iteration of each mask bit
  LiveGroup live[2][2];
  bool live_open[2][2] = {};
  uint64_t live_ticket[2][2][64] = {};
  uint32_t live_iter0[2][2][64] = {};
  // Groups of one algorithm on the device at once.  A second group (for the
  // arrivals after the first one's join window) measured slower at
  // RMAT-26 edge factor 48: 72.9 against 90.2 q/s at 32x the single-run
  // capacity, p50 1.41 against 0.96 s at 4x: turns between two groups delay
  // both.
  uint32_t groups_per_algo = 1;
};

namespace {

double clock_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

void server_free(thv_server *s) {
  for (int k = 0; k < 2; k++)
    for (int i = 0; i < 2; i++)
      if (s->live_open[k][i]) live_close(&s->live[k][i]);
  dev_free(s->d_val);
  dev_free(s->d_bm);
  dev_free(s->d_out);
  dev_free(s->d_front);
  dev_free(s->d_qsm);
  dev_free(s->d_qbm);
  dev_free(s->d_sum);
  dev_free(s->d_qs);
  dev_free(s->d_qb);
  dev_free(s->d_ctrl);
  pinned_free(s->h_ctrl);
  dev_free(s->d_seeds);
  pinned_free(s->h_seeds);
  pinned_free(s->h_sum);
  if (s->st) cudaStreamDestroy(s->st);
}

SvArgs make_args(thv_server *s) {
  thv_graph *g = s->g;
  SvArgs a{};
  a.off = g->d_off;
  a.blk_vb = g->plan.d_vbegin;
  a.blk_base = g->plan.d_base;
  a.host_base = g->h_edges_dev;
  a.lc = list_cache_of(g->plan);
  a.blk_access = g->plan.d_access;
  // 4-byte edges: packed weights, or unit weights for an unweighted graph
  a.wshift = g->wshift;
  a.wbase = g->packed ? g->wbase : 1u;
  a.val = s->d_val;
  a.front = s->d_front;
  a.bm = s->d_bm;
  a.qs = s->d_qs;
  a.qb = s->d_qb;
  a.qsm = s->d_qsm;
  a.qbm = s->d_qbm;
  a.cap_s = s->cap_s;
  a.cap_b = s->cap_b;
  a.ctrl = s->d_ctrl;
  a.timeout_ns = s->timeout_ns;
  a.nblk = (uint32_t)g->plan.blocks.size();
  a.nv = (uint32_t)g->nv;
  a.ngroups = s->ngroups;
  a.W = s->W;
  a.small_deg = 64;
  a.chunk = 256;
  return a;
}

// One launch of the serving kernel; returns the finished-slot mask.
thv_status step(thv_server *s, uint32_t max_iters, unsigned long long *done, uint32_t *iters) {
  thv_graph *g = s->g;
  SvArgs a = make_args(s);
  a.active = s->active;
  a.unit = s->unit;
  a.max_iters = max_iters;
  const size_t smem = g->plan.vbegin.size() <= kSmemBlocks + 1 ? g->plan.vbegin.size() * 4 : 0;
  void *kern = g->esz == 8 ? (void *)sv_kernel<8> : (void *)sv_kernel<4>;
  int bpsm = 0;
  if (g->esz == 8)
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, sv_kernel<8>, kSvThreads, smem));
  else
    THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, sv_kernel<4>, kSvThreads, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "serving kernel cannot be resident");
  // the rotating per-iteration counters restart with every launch
  const size_t c0 = offsetof(SvCtrl, cnt_small), c1 = offsetof(SvCtrl, thr);
  THV_CUDA(cudaMemsetAsync((char *)s->d_ctrl + c0, 0, c1 - c0, s->st));
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel(kern, dim3(bpsm * g->num_sms), dim3(kSvThreads), args, smem, s->st));
  THV_CUDA(cudaMemcpyAsync(s->h_ctrl, s->d_ctrl, sizeof(SvCtrl), cudaMemcpyDeviceToHost, s->st));
  THV_CUDA(cudaStreamSynchronize(s->st));
  const SvCtrl &hc = *s->h_ctrl;
  if (hc.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "serving: grid barrier timeout");
  if (hc.err) return fail(THV_EDEVICE, "serving: device error %u", hc.err);
  *done = hc.done_mask;
  *iters = hc.iters;
  return THV_OK;
}

thv_status retire(thv_server *s, unsigned long long done) {
  thv_graph *g = s->g;
  SvArgs a = make_args(s);
  const int grid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  while (done) {
    const int slot = __builtin_ctzll(done);
    done &= done - 1;
    uint64_t ticket;
    uint32_t *out;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      ticket = s->slot_ticket[slot];
      out = s->queries[ticket].out;
    }
    THV_CUDA(cudaMemsetAsync(s->d_sum, 0, 8, s->st));
    sv_extract<<<grid, 256, 0, s->st>>>(a, (uint32_t)slot, out ? s->d_out : nullptr, s->d_sum);
    THV_CUDA(cudaGetLastError());
    THV_CUDA(cudaMemcpyAsync(s->h_sum, s->d_sum, 8, cudaMemcpyDeviceToHost, s->st));
    if (out) THV_CUDA(cudaMemcpyAsync(out, s->d_out, g->nv * 4, cudaMemcpyDeviceToHost, s->st));
    THV_CUDA(cudaStreamSynchronize(s->st));
    std::lock_guard<std::mutex> lk(s->mu);
    Query &q = s->queries[ticket];
    q.checksum = *s->h_sum;
    q.t_done = clock_ms();
    q.iterations = (uint32_t)(s->total_iters - q.iter_start);
    q.done = true;
    s->active &= ~(1ull << slot);
    s->unit &= ~(1ull << slot);
    s->slot_ticket[slot] = 0;
    s->done_since_replan++;
  }
  s->cv_done.notify_all();
  return THV_OK;
}

void fail_all(thv_server *s, thv_status st, const std::string &msg) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->fatal = st;
  s->fatal_msg = msg;
  for (auto &kv : s->queries) {
    if (!kv.second.done) {
      kv.second.done = true;
      kv.second.status = st;
      kv.second.t_done = clock_ms();
    }
  }
  s->waiting.clear();
  s->active = 0;
  s->cv_done.notify_all();
}

// Iterations per launch of a live group: one while anything waits to join
// or the other algorithm's group shares the device (so admission and the
// turns stay short), else thv_serve_opts.max_batch_iters (default 4: fewer
// returns to the host).
constexpr uint32_t kLiveItersBusy = 1;

// Adds tickets (all of algorithm k) to live group (k, i), opening it on
// first use.
thv_status live_join(thv_server *s, int k, int i, const std::vector<uint64_t> &tickets) {
  if (tickets.empty()) return THV_OK;
  thv_graph *g = s->g;
  LiveGroup &lg = s->live[k][i];
  if (!s->live_open[k][i]) {
    s->live_open[k][i] = true;  // live_close frees whatever live_open allocated
    THV_TRY(live_open(g, &lg, k == 1));
  }
  std::vector<uint32_t> src(tickets.size()), bits(tickets.size());
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t j = 0; j < tickets.size(); j++) src[j] = s->queries[tickets[j]].source;
  }
  THV_TRY(live_add(g, &lg, (uint32_t)src.size(), src.data(), bits.data(),
                   (uint32_t)(s->timeout_ns / 1000000ull), s->st));
  std::lock_guard<std::mutex> lk(s->mu);
  for (size_t j = 0; j < tickets.size(); j++) {
    s->live_ticket[k][i][bits[j]] = tickets[j];
    s->live_iter0[k][i][bits[j]] = lg.iter;
    s->queries[tickets[j]].slot = bits[j];
  }
  return THV_OK;
}

thv_status run_alone(thv_server *s, thv_algo algo, uint64_t ticket);

// One launch of live group (k, i), then its finished sources' results.
thv_status live_turn(thv_server *s, int k, int i, uint32_t iters) {
  LiveGroup &lg = s->live[k][i];
  unsigned long long fin = 0;
  bool too_deep = false;
  const uint32_t tmo = (uint32_t)(s->timeout_ns / 1000000ull);
  THV_TRY(live_step(s->g, &lg, iters, tmo, s->st, &fin, &too_deep));
  if (too_deep) {
    // a BFS level left the u8 range: its queries run alone instead
    std::vector<uint64_t> redo;
    for (unsigned long long m = lg.active; m; m &= m - 1) redo.push_back(s->live_ticket[k][i][__builtin_ctzll(m)]);
    lg.active = 0;
    lg.running = false;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (uint64_t t : redo) s->queries[t].mode = 2;
    }
    for (uint64_t t : redo) THV_TRY(run_alone(s, k ? THV_ALGO_SSSP : THV_ALGO_BFS, t));
    return THV_OK;
  }
  if (!fin) return THV_OK;
  uint32_t *outs[64] = {};
  uint64_t sums[64] = {};
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (unsigned long long m = fin; m; m &= m - 1) {
      const int b = __builtin_ctzll(m);
      outs[b] = s->queries[s->live_ticket[k][i][b]].out;
    }
  }
  THV_TRY(live_collect(s->g, &lg, fin, sums, outs, s->d_out, s->st));
  std::lock_guard<std::mutex> lk(s->mu);
  const double now = clock_ms();
  for (unsigned long long m = fin; m; m &= m - 1) {
    const int b = __builtin_ctzll(m);
    Query &q = s->queries[s->live_ticket[k][i][b]];
    q.checksum = sums[b];
    q.t_done = now;
    q.iterations = lg.iter - s->live_iter0[k][i][b];
    q.status = THV_OK;
    q.done = true;
    s->live_ticket[k][i][b] = 0;
    s->done_since_replan++;
  }
  s->cv_done.notify_all();
  return THV_OK;
}

// One query on the single-source kernel (values into its buffer, checksum).
thv_status run_alone(thv_server *s, thv_algo algo, uint64_t ticket) {
  uint32_t source;
  uint32_t *out;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const Query &q = s->queries[ticket];
    source = q.source;
    out = q.out;
  }
  thv_run_opts ro{};
  ro.source = source;
  ro.timeout_ms = (uint32_t)(s->timeout_ns / 1000000ull);
  ro.flags = THV_RUN_CHECKSUM;
  thv_stats st1{};
  thv_status st = run_minprop(s->g, algo, &ro, s->st, &st1);
  if (st == THV_OK && out) st = minprop_values(s->g, out, s->st);
  std::lock_guard<std::mutex> lk(s->mu);
  Query &q = s->queries[ticket];
  q.checksum = st1.checksum;
  q.t_done = clock_ms();
  q.iterations = (uint32_t)st1.iterations;
  q.slot = 0;
  q.status = st;
  q.done = true;
  s->total_iters += st1.iterations;
  s->done_since_replan++;
  s->cv_done.notify_all();
  return st;
}

bool live_running(const thv_server *s, int k) {
  return s->live[k][0].running || s->live[k][1].running;
}
bool live_running(const thv_server *s) { return live_running(s, 0) || live_running(s, 1); }

// Batching mode, one dispatcher round.  Admission, per algorithm: a running
// group still inside its join window (its first join_window iterations)
// takes waiting queries into free mask bits -- sources that start within a
// couple of levels of each other share most edge reads; otherwise a new
// group starts when enough queries wait (group_min), or at once when no
// group of this algorithm runs but the other algorithm's does (they share
// the device by turns anyway), up to groups_per_algo groups, so arrivals
// need not wait for an old group to drain.  With nothing on the device and
// too few waiting, the front query runs alone.  Then every running group
// gets one turn.
thv_status batching_round(thv_server *s) {
  std::vector<uint64_t> joins[2][2];
  uint64_t alone = 0;
  thv_algo alone_algo = THV_ALGO_BFS;
  bool waiting_for[2] = {false, false};
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const double now = clock_ms();
    for (int k = 0; k < 2; k++) {
      const thv_algo algo = k ? THV_ALGO_SSSP : THV_ALGO_BFS;
      uint32_t n = 0;
      for (uint64_t t : s->waiting) n += s->queries[t].algo == algo;
      if (!n) continue;
      int inst = -1;
      uint32_t take = 0;
      bool joined = false;
      for (int i = 0; i < (int)s->groups_per_algo && inst < 0; i++) {
        LiveGroup &lg = s->live[k][i];
        if (lg.running && live_can_join(s->g, &lg) && (!s->join_window || lg.iter < s->join_window)) {
          inst = i;
          take = std::min<uint32_t>(n, kGroupMax - __builtin_popcountll(lg.active));
          joined = true;
        }
      }
      if (inst < 0) {
        const uint32_t kmin = s->group_min ? s->group_min : (k ? kGroupMinSssp : kGroupMinBfs);
        const bool any_k = live_running(s, k);
        for (int i = 0; i < (int)s->groups_per_algo && inst < 0; i++) {
          if (s->live[k][i].running) continue;
          if (n >= kmin || (!any_k && live_running(s, 1 - k))) {
            inst = i;
            take = std::min<uint32_t>(n, kGroupMax);
          }
        }
      }
      waiting_for[k] = take < n;
      if (inst < 0) continue;
      std::vector<uint64_t> &jv = joins[k][inst];
      for (auto it = s->waiting.begin(); it != s->waiting.end() && jv.size() < take;) {
        Query &q = s->queries[*it];
        if (q.algo != algo) {
          ++it;
          continue;
        }
        q.t_start = now;
        q.mode = 1;
        q.joined = joined;
        jv.push_back(*it);
        it = s->waiting.erase(it);
      }
    }
    bool any_join = false;
    for (int k = 0; k < 2; k++)
      for (int i = 0; i < 2; i++) any_join |= !joins[k][i].empty();
    if (!any_join && !live_running(s) && !s->waiting.empty()) {
      alone = s->waiting.front();
      s->waiting.pop_front();
      Query &q = s->queries[alone];
      q.t_start = clock_ms();
      q.mode = 2;
      alone_algo = q.algo;
    }
  }
  if (alone) return run_alone(s, alone_algo, alone);
  for (int k = 0; k < 2; k++)
    for (int i = 0; i < 2; i++) THV_TRY(live_join(s, k, i, joins[k][i]));
  int nrunning = 0;
  for (int k = 0; k < 2; k++)
    for (int i = 0; i < 2; i++) nrunning += s->live[k][i].running;
  for (int k = 0; k < 2; k++) {
    for (int i = 0; i < 2; i++) {
      if (!s->live[k][i].running) continue;
      bool waits;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        waits = !s->waiting.empty();
      }
      const uint32_t iters = nrunning > 1 || waits || waiting_for[k] ? kLiveItersBusy : s->batch_iters;
      THV_TRY(live_turn(s, k, i, iters));
    }
  }
  return THV_OK;
}

void worker_loop(thv_server *s) {
  cudaSetDevice(s->g->device);
  for (;;) {
    uint32_t nseed = 0;
    bool requests_waiting = false;
    uint64_t lone = 0;
    thv_algo lone_algo = THV_ALGO_BFS;
    bool replan = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] {
        return s->stopping || !s->waiting.empty() || s->active || live_running(s);
      });
      if (s->stopping && s->waiting.empty() && !s->active && !live_running(s)) return;
      // between queries (nothing on the device), re-place the edge blocks by
      // the access this server measured
      if (s->replan_every && !s->active && !live_running(s) &&
          s->done_since_replan >= s->replan_every && (s->g->plan.flags & THV_PLAN_TRACK_ACCESS)) {
        s->done_since_replan = 0;
        replan = true;
      }
    }
    if (replan) {
      const thv_status st = replan_by_access(s->g);
      if (st != THV_OK) {
        fail_all(s, st, thv_last_error());
        return;
      }
      continue;
    }
    if (s->batching) {
      const thv_status st = batching_round(s);
      if (st != THV_OK) {
        fail_all(s, st, thv_last_error());
        return;
      }
      continue;
    }
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // Slots: an idle server with one request runs it on the single-source
      // kernel; otherwise each waiting query takes a free slot (its column
      // was reset when the slot's last query retired).
      if (!s->active && s->waiting.size() == 1) {
        lone = s->waiting.front();
        s->waiting.pop_front();
        Query &q = s->queries[lone];
        lone_algo = q.algo;
        q.t_start = clock_ms();
        q.mode = 2;
      }
      while (!lone && !s->waiting.empty()) {
        int slot = -1;
        for (uint32_t i = 0; i < s->W; i++)
          if (!((s->active >> i) & 1ull)) { slot = (int)i; break; }
        if (slot < 0) break;
        const uint64_t t = s->waiting.front();
        s->waiting.pop_front();
        Query &q = s->queries[t];
        q.slot = (uint32_t)slot;
        q.t_start = clock_ms();
        q.iter_start = (uint32_t)s->total_iters;
        q.joined = s->active != 0;
        const bool bfs = q.algo == THV_ALGO_BFS;
        s->h_seeds[nseed++] = SvSeed{(uint32_t)slot, q.source, bfs ? 2u : 1u + kSvDeltaSssp,
                                     bfs ? 1u : kSvDeltaSssp};
        s->active |= 1ull << slot;
        if (bfs) s->unit |= 1ull << slot;
        s->slot_ticket[slot] = t;
      }
      // with a free slot, return to the host every few iterations so that a
      // request arriving meanwhile is admitted quickly; with none free, run
      // until a query finishes
      requests_waiting = __builtin_popcountll(s->active) < (int)s->W;
    }
    if (lone) {
      const thv_status st = run_alone(s, lone_algo, lone);
      if (st != THV_OK) {
        fail_all(s, st, thv_last_error());
        return;
      }
      continue;
    }
    if (nseed) {
      SvArgs a = make_args(s);
      if (cudaMemcpyAsync(s->d_seeds, s->h_seeds, nseed * sizeof(SvSeed), cudaMemcpyHostToDevice,
                          s->st) != cudaSuccess) {
        fail_all(s, THV_ECUDA, "seed copy failed");
        return;
      }
      sv_seed<<<1, kSvMaxSlots, 0, s->st>>>(a, s->d_seeds, nseed);
    }
    unsigned long long done = 0;
    uint32_t iters = 0;
    const uint32_t budget = requests_waiting ? s->batch_iters : 1u << 20;
    thv_status st = step(s, budget, &done, &iters);
    if (st != THV_OK) {
      fail_all(s, st, thv_last_error());
      return;
    }
    s->total_iters += iters;
    if (done && (st = retire(s, done)) != THV_OK) {
      fail_all(s, st, thv_last_error());
      return;
    }
  }
}

thv_status start(thv_graph *g, const thv_serve_opts *o, thv_server **out) {
  if (g->fmt == THV_FMT_CSC) return fail(THV_EINVAL, "serving needs out-edges (CSR/WCSR)");
  if (g->nv >= 0xFFFFFFFFull) return fail(THV_EUNSUPPORTED, "too many vertices");
  THV_TRY(ensure_plan(g));
  std::unique_ptr<thv_server, void (*)(thv_server *)> s(new thv_server(), [](thv_server *p) {
    server_free(p);
    delete p;
  });
  s->g = g;
  uint32_t W = o && o->max_slots ? std::min<uint32_t>(o->max_slots, kSvMaxSlots) : kSvMaxSlots;
  if (o && o->mem_budget_bytes) {
    const uint64_t per_slot = g->nv * 4ull;
    W = (uint32_t)std::min<uint64_t>(W, o->mem_budget_bytes / per_slot);
    if (W == 0) return fail(THV_ENOMEM, "memory budget %llu below one slot (%llu bytes)",
                            (unsigned long long)o->mem_budget_bytes, (unsigned long long)per_slot);
  }
  s->W = W;
  s->queue_cap = o && o->queue_capacity ? o->queue_capacity : 65536u;
  s->batch_iters = o && o->max_batch_iters ? o->max_batch_iters : 4u;
  s->batching = !(o && o->group_min == 0xFFFFFFFFu);
  s->group_min = o && o->group_min && o->group_min != 0xFFFFFFFFu ? o->group_min : 0u;
  s->replan_every = o ? o->replan_every : 0;
  s->join_window = o && o->join_window ? (o->join_window == 0xFFFFFFFFu ? 0u : o->join_window)
                                       : kJoinWindow;
  s->groups_per_algo = o && o->groups_per_algo ? std::min<uint32_t>(o->groups_per_algo, 2u) : 1u;
  if (o && o->mem_budget_bytes && o->mem_budget_bytes < g->nv * kGroupBytesPerVertex)
    s->batching = false;  // the batch state does not fit the memory budget
  s->timeout_ns = (uint64_t)(o && o->timeout_ms ? o->timeout_ms : 60000u) * 1000000ull;
  THV_TRY(dev_alloc((void **)&s->d_out, g->nv * 4 + 64, "serving output"));
  THV_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  if (s->batching) {
    // live groups allocate their batch state on first use
    thv_server *raw = s.release();
    raw->worker = std::thread(worker_loop, raw);
    *out = raw;
    return THV_OK;
  }
  const uint64_t nw = (g->nv + 31) / 32;
  s->ngroups = (uint32_t)((nw + 31) / 32);
  const uint64_t nw_alloc = (uint64_t)s->ngroups * 32;
  s->cap_s = g->nv + 32;
  s->cap_b = g->ne / 256 + g->ne / 64 + 64;
  THV_TRY(dev_alloc((void **)&s->d_val, g->nv * (uint64_t)W * 4 + 64, "serving values"));
  THV_TRY(dev_alloc((void **)&s->d_front, g->nv * 8 + 64, "serving masks"));
  THV_TRY(dev_alloc((void **)&s->d_bm, nw_alloc * 4, "serving bitmap"));
  THV_TRY(dev_alloc((void **)&s->d_qs, s->cap_s * sizeof(WorkItem), "serving queue"));
  THV_TRY(dev_alloc((void **)&s->d_qsm, s->cap_s * 8, "serving queue masks"));
  THV_TRY(dev_alloc((void **)&s->d_qb, s->cap_b * sizeof(WorkItem), "serving chunk queue"));
  THV_TRY(dev_alloc((void **)&s->d_qbm, s->cap_b * 8, "serving chunk masks"));
  THV_TRY(dev_alloc((void **)&s->d_ctrl, sizeof(SvCtrl), "serving control"));
  THV_TRY(pinned_alloc((void **)&s->h_ctrl, sizeof(SvCtrl), "serving control"));
  THV_TRY(dev_alloc((void **)&s->d_seeds, kSvMaxSlots * sizeof(SvSeed), "serving seeds"));
  THV_TRY(pinned_alloc((void **)&s->h_seeds, kSvMaxSlots * sizeof(SvSeed), "serving seeds"));
  THV_TRY(dev_alloc((void **)&s->d_sum, 8, "serving checksum"));
  THV_TRY(pinned_alloc((void **)&s->h_sum, 8, "serving checksum"));
  SvArgs a = make_args(s.get());
  const int grid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  sv_reset<<<grid, 256, 0, s->st>>>(a, (uint32_t)nw_alloc);
  THV_CUDA(cudaGetLastError());
  THV_CUDA(cudaStreamSynchronize(s->st));
  thv_server *raw = s.release();
  raw->worker = std::thread(worker_loop, raw);
  *out = raw;
  return THV_OK;
}

}  // namespace

extern "C" {

thv_status thv_serve_start(thv_graph *g, const thv_serve_opts *o, thv_server **out) {
  try {
    if (!g || !out) return fail(THV_EINVAL, "null argument");
    THV_CUDA(cudaSetDevice(g->device));
    return start(g, o, out);
  } catch (...) {
    return fail(THV_ENOMEM, "serving start: host allocation failed");
  }
}

thv_status thv_serve_submit(thv_server *s, thv_algo algo, uint32_t source, uint32_t *out,
                            uint64_t *ticket) {
  if (!s || !ticket) return fail(THV_EINVAL, "null argument");
  if (algo != THV_ALGO_BFS && algo != THV_ALGO_SSSP)
    return fail(THV_EINVAL, "serving runs BFS and SSSP queries");
  if (algo == THV_ALGO_SSSP && !s->g->weighted) return fail(THV_EINVAL, "SSSP needs edge weights");
  if (source >= s->g->nv) return fail(THV_EINVAL, "source %u out of range", source);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->fatal != THV_OK) return fail(s->fatal, "server failed: %s", s->fatal_msg.c_str());
  if (s->stopping) return fail(THV_EINVAL, "server is stopping");
  if (s->waiting.size() >= s->queue_cap) return fail(THV_EBUSY, "serving queue full");
  const uint64_t t = s->next_ticket++;
  Query q;
  q.algo = algo;
  q.source = source;
  q.out = out;
  q.t_submit = clock_ms();
  s->queries.emplace(t, q);
  s->waiting.push_back(t);
  *ticket = t;
  s->cv_work.notify_one();
  return THV_OK;
}

static thv_status collect(thv_server *s, uint64_t ticket, thv_query_stats *st) {
  auto it = s->queries.find(ticket);
  if (it == s->queries.end()) return fail(THV_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
  if (!it->second.done) return THV_ENOTREADY;
  const Query &q = it->second;
  if (st) {
    st->queue_ms = q.t_start > 0 ? q.t_start - q.t_submit : 0;
    st->run_ms = q.t_start > 0 ? q.t_done - q.t_start : 0;
    st->latency_ms = q.t_done - q.t_submit;
    st->checksum = q.checksum;
    st->iterations = q.iterations;
    st->slot = q.slot;
    st->status = q.status;
    st->grouped = q.mode;
    st->joined = q.joined ? 1u : 0u;
    st->pad = 0;
  }
  const thv_status qs = q.status;
  s->queries.erase(it);
  return qs == THV_OK ? THV_OK : fail(qs, "query failed");
}

thv_status thv_serve_poll(thv_server *s, uint64_t ticket, thv_query_stats *st) {
  if (!s) return fail(THV_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  return collect(s, ticket, st);
}

thv_status thv_serve_wait(thv_server *s, uint64_t ticket, thv_query_stats *st, uint32_t timeout_ms) {
  if (!s) return fail(THV_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] {
    auto it = s->queries.find(ticket);
    return it == s->queries.end() || it->second.done;
  };
  if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms ? timeout_ms : 60000), ready))
    return fail(THV_ETIMEOUT, "query %llu not done", (unsigned long long)ticket);
  return collect(s, ticket, st);
}

thv_status thv_serve_stop(thv_server *s) {
  if (!s) return THV_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  const thv_status st = s->fatal;
  cudaSetDevice(s->g->device);
  server_free(s);
  delete s;
  return st == THV_OK ? THV_OK : fail(st, "server had failed");
}

}  // extern "C"
