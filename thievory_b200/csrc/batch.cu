// Batched multi-source BFS / SSSP: up to 64 sources share one traversal.
//
// No counterpart in the reference (it runs one source per process,
// src/bfs/bfs.cu:8, src/sssp/sssp.cu:10).  Same frontier machinery as the
// single-source engine (minprop.cu) -- pending-vertex bitmap, ballot
// compaction into small-vertex groups and high-degree chunks, zero-copy
// addressing of non-resident blocks -- but every vertex carries a 64-bit
// mask of the sources for which it is pending, and each work item carries
// the mask it was taken with, so ONE read of an adjacency list serves all
// the sources that need it:
//   BFS  (MS-BFS): visit[v] is the set of sources that reached v.  An edge
//        u->w with frontier mask f does m = f & ~visit[w]; atomicOr(visit[w],
//        m) hands each newly reached (w, s) to exactly one thread, which
//        writes level byte lvl[w][s] = iteration + 1 and marks w pending.
//   SSSP dist[w][.] rows of 64 u32 (vertex-major, one 256-byte row per
//        vertex; source s at word row_pos(s)); per edge and source in the
//        mask the single-source
//        relaxation "cand < dist => atomicMin, mark pending" with the same
//        near/far window, shared by all sources.
// Results are bit-identical to single-source runs: BFS levels are exact
// (level-synchronous), SSSP is the unique min fixed point.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

enum { MS_BFS = 0, MS_SSSP = 1 };
constexpr uint32_t kMsWidth = 64;       // sources per group (mask bits)
constexpr uint32_t kMaxBfsLevel = 254;  // u8 level bytes hold level + 1
constexpr uint32_t kMsGrowth = 1;       // SSSP window width factor per advance
constexpr uint32_t kMsDelta = 256;      // SSSP window width shared by a group
// SSSP: steps (two edges, one 16-byte row piece per lane each) whose rows
// are in flight at once, staged through a per-warp shared-memory ring by
// asynchronous copies (64 KiB per 512-thread block; 12 and 16 measured
// slower at RMAT-26)
constexpr uint32_t kMsRing = 8;

// Word of source s in a 64-word SSSP distance row: lane l of a half-warp
// holds sources l, l+16, l+32, l+48 as one 16-byte word group (4l..4l+3),
// so one 16-byte load per lane reads a whole row per half-warp.
__host__ __device__ __forceinline__ uint32_t row_pos(uint32_t s) {
  return 4u * (s & 15u) + (s >> 4);
}

struct MsCtrl {
  GridBar bar;
  unsigned err, iters;
  unsigned long long cnt_small[3], cnt_big[3], remaining[3], wc[3];
  unsigned minkept[3], pad;
  unsigned long long edges, hbm_bytes, link_bytes, pairs;
  // live groups: where a launch that yielded stopped (the next launch
  // resumes there), and the OR of the pending-source masks after it
  unsigned y_iter, y_level, y_thr, y_width, yielded, pad2;
  unsigned long long alive;
  unsigned long long cnt_mid[3];  // kept off the line of the barrier and hot counters
};

struct MsArgs {
  const uint64_t *off;
  const uint32_t *blk_vb;
  const uint64_t *blk_base;
  uint64_t host_base;
  ListCache lc;
  unsigned long long *blk_access;  // tracked plans: adjacency bytes read per block
  unsigned long long *visit;  // BFS
  unsigned long long *front;  // pending (vertex, source) pairs
  uint8_t *lvl;               // BFS [nv][64]: level + 1, 0 = unreached
  uint32_t *dist;             // SSSP [nv][64]: distance + 1
  uint32_t *bm;
  uint32_t *wmin;             // SSSP: lower bound of pending distances per word
  WorkItem *qs, *qb, *qm;
  unsigned long long *qsm, *qbm, *qmm;  // masks of the queued items
  unsigned long long cap_s, cap_b;
  MsCtrl *ctrl;
  const uint32_t *sources;  // [k, source 0, ..., source k-1]
  unsigned long long timeout_ns;
  uint32_t nblk, nv, ngroups, max_iters;
  // degree buckets: [1, small_deg) in groups of gsmall vertices per warp,
  // [small_deg, mid_deg) in groups of gmid, the rest in chunk-edge items
  uint32_t small_deg, chunk, delta;
  uint32_t mid_deg, gsmall, gmid;
  uint32_t wshift, wbase;  // packed weighted edges (see edge_dst / edge_wt)
  uint32_t growth;         // SSSP window width factor per advance
  // live groups: a launch returns at the top of iteration yield_at (0 =
  // run to completion); resume = 1 starts from r_* instead of iteration 0
  uint32_t yield_at, resume;
  uint32_t r_iter, r_level, r_thr, r_width;
};

struct BatchState {
  uint64_t nv = 0;
  bool sssp = false;
  bool valid = false;  // every allocation succeeded
  unsigned long long *d_visit = nullptr, *d_front = nullptr;
  uint8_t *d_lvl = nullptr;
  uint32_t *d_dist = nullptr;
  uint32_t *d_bm = nullptr, *d_wmin = nullptr;
  WorkItem *d_qs = nullptr, *d_qb = nullptr, *d_qm = nullptr;
  unsigned long long *d_qsm = nullptr, *d_qbm = nullptr, *d_qmm = nullptr;
  uint64_t cap_s = 0, cap_b = 0;
  MsCtrl *d_ctrl = nullptr, *h_ctrl = nullptr;
  uint32_t *d_sources = nullptr, *h_sources = nullptr;
  uint32_t *d_out = nullptr;  // kMsWidth x nv u32 staging for host output
  unsigned long long *d_sums = nullptr, *h_sums = nullptr;
  uint32_t ngroups = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

// ---------------------------------------------------------------- device --

template <int OP>
__device__ __forceinline__ void mark_pending(const MsArgs &a, uint32_t w) {
  const uint32_t m = 1u << (w & 31u);
  uint32_t *bp = a.bm + (w >> 5);
  if (!(ldcg(bp) & m)) atomicOr(bp, m);
}

// BFS edge u->w for the sources in f, discovered at level `lvl1` (= L + 1).
__device__ __forceinline__ void ms_bfs_edge(const MsArgs &a, uint32_t w,
                                            unsigned long long f, uint32_t lvl1) {
  const unsigned long long m = f & ~ldcg(a.visit + w);
  if (!m) return;
  const unsigned long long old = atomicOr(a.visit + w, m);
  unsigned long long nb = m & ~old;
  if (!nb) return;
  atomicOr(a.front + w, nb);
  mark_pending<MS_BFS>(a, w);
  uint8_t *row = a.lvl + (size_t)w * kMsWidth;
  while (nb) {
    const int s = __ffsll((long long)nb) - 1;
    nb &= nb - 1;
    row[s] = (uint8_t)lvl1;
  }
}

// BFS edges w[j] for the source masks f[j] (0: no edge), N per lane: the
// visit probes, then the claiming atomicOr's, are issued for all N edges
// before any result is used, so a lane has N requests in flight per step.
template <int N>
__device__ __forceinline__ void ms_bfs_edges(const MsArgs &a, const uint32_t (&w)[N],
                                             const unsigned long long (&f)[N], uint32_t lvl1) {
  unsigned long long m[N];
#pragma unroll
  for (int j = 0; j < N; j++) m[j] = f[j] ? f[j] & ~ldcg(a.visit + w[j]) : 0ull;
#pragma unroll
  for (int j = 0; j < N; j++) m[j] = m[j] ? m[j] & ~atomicOr(a.visit + w[j], m[j]) : 0ull;
#pragma unroll
  for (int j = 0; j < N; j++) {
    unsigned long long nb = m[j];
    if (!nb) continue;
    atomicOr(a.front + w[j], nb);
    mark_pending<MS_BFS>(a, w[j]);
    uint8_t *row = a.lvl + (size_t)w[j] * kMsWidth;
    while (nb) {
      const int s = __ffsll((long long)nb) - 1;
      nb &= nb - 1;
      row[s] = (uint8_t)lvl1;
    }
  }
}

// SSSP edge u->w of weight wt for the sources in f.  The distance update
// is a fire-and-forget atomicMin: when cand is below the value read, (w, s)
// is marked pending whether this lane or a concurrent one ends up lowering
// dist[w][s] (the lower writer marks the same bit in the same phase), so
// the lane never waits for the old value.
__device__ __forceinline__ void ms_sssp_edge(const MsArgs &a, uint32_t u, uint32_t w,
                                             uint32_t wt, unsigned long long f) {
  const uint32_t *du = a.dist + (size_t)u * kMsWidth;
  uint32_t *dw = a.dist + (size_t)w * kMsWidth;
  unsigned long long improved = 0;
  uint32_t best = 0xFFFFFFFFu;
  while (f) {
    const int s = __ffsll((long long)f) - 1;
    f &= f - 1;
    const uint32_t p = row_pos((uint32_t)s);
    const unsigned long long cand = (unsigned long long)ldcg(du + p) + wt;
    if (cand < ldcg(dw + p)) {
      atomicMin(dw + p, (uint32_t)cand);
      improved |= 1ull << s;
      best = min(best, (uint32_t)cand);
    }
  }
  if (improved) {
    atomicOr(a.front + w, improved);
    atomicMin(a.wmin + (w >> 5), best);
    mark_pending<MS_SSSP>(a, w);
  }
}

// 16-byte asynchronous global -> shared copy (L2 only); a false `ok`
// zero-fills the destination without reading.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool ok) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(ok ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}

// Half-warp-per-edge SSSP relaxation of one work item: the warp loads the
// item's edges 32 at a time (coalesced); each half-warp takes one edge and
// reads its whole 256-byte distance row, one 16-byte piece per lane (lane
// l: sources l, l+16, l+32, l+48), so a warp step relaxes two edges for all
// 64 sources.  The row pieces go through `ring` (this lane's slot of the
// warp's kMsRing x 512-byte shared ring) by asynchronous copies issued
// kMsRing steps ahead, so 2 x kMsRing rows are in flight without holding
// registers.  Each lane reads back only the piece it copied itself.
// Distance updates are fire-and-forget as in ms_sssp_edge; four ballots
// give each edge's improved-source mask.
template <int ESZ>
__device__ __forceinline__ void ms_sssp_item(const MsArgs &a, uint32_t ring, uint32_t u,
                                             uintptr_t eaddr, uint32_t cnt, unsigned long long f) {
  const unsigned lane = lane_id(), hl = lane & 15u, half = lane >> 4;
  const uint32_t mb = (uint32_t)((f >> hl) & 1ull) | (uint32_t)((f >> (hl + 15u)) & 2ull) |
                      (uint32_t)((f >> (hl + 30u)) & 4ull) | (uint32_t)((f >> (hl + 45u)) & 8ull);
  uint4 du4 = make_uint4(0, 0, 0, 0);
  if (mb) du4 = __ldcg(reinterpret_cast<const uint4 *>(a.dist + (size_t)u * kMsWidth) + hl);
  const uint32_t du[4] = {du4.x, du4.y, du4.z, du4.w};
  for (uint32_t base = 0; base < cnt; base += 32) {
    // packed edges stay raw until used
    uint2 e = make_uint2(0, 0);
    if (base + lane < cnt) {
      if (ESZ == 8) e = ld_nc_u2(eaddr + (uintptr_t)(base + lane) * 8u);
      else e.x = ld_nc_u32(eaddr + (uintptr_t)(base + lane) * 4u);
    }
    const uint32_t m = min(32u, cnt - base), nsteps = (m + 1) / 2;
    // step st: edges 2st (lanes 0-15) and 2st+1 (lanes 16-31); one copy
    // group per step, empty past the end, so group st completes step st
    auto issue = [&](uint32_t st) {
      if (st < nsteps) {
        const uint32_t idx = 2u * st + half;
        const uint32_t x = __shfl_sync(kFull, e.x, idx & 31u);
        const uint32_t w = ESZ == 8 ? x : edge_dst(x, a.wshift);
        const bool ok = idx < m && mb;
        cp_async16(ring + (st % kMsRing) * 512u,
                   ok ? (const void *)(a.dist + (size_t)w * kMsWidth + 4u * hl) : (const void *)a.dist,
                   ok);
      }
      cp_async_commit();
    };
#pragma unroll
    for (uint32_t st = 0; st < kMsRing; st++) issue(st);
    for (uint32_t st = 0; st < nsteps; st++) {
      cp_async_wait<kMsRing - 1>();
      const uint4 dw = lds128(ring + (st % kMsRing) * 512u);
      const uint32_t idx = 2u * st + half;
      const uint32_t x = __shfl_sync(kFull, e.x, idx & 31u);
      const uint32_t y = ESZ == 8 ? __shfl_sync(kFull, e.y, idx & 31u) : 0u;
      const bool ok = idx < m;
      const uint32_t w = ESZ == 8 ? x : edge_dst(x, a.wshift);
      const uint32_t wt = ESZ == 8 ? y : edge_wt(x, a.wshift, a.wbase);
      uint32_t *row = a.dist + (size_t)w * kMsWidth + 4u * hl;
      const uint32_t cw[4] = {dw.x, dw.y, dw.z, dw.w};
      uint32_t imp = 0, best = 0xFFFFFFFFu;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const unsigned long long cand = (unsigned long long)du[i] + wt;
        if (ok && ((mb >> i) & 1u) && cand < cw[i]) {
          atomicMin(row + i, (uint32_t)cand);
          imp |= 1u << i;
          best = min(best, (uint32_t)cand);
        }
      }
      if (__any_sync(kFull, imp != 0)) {
        const unsigned b0 = __ballot_sync(kFull, imp & 1u), b1 = __ballot_sync(kFull, imp & 2u);
        const unsigned b2 = __ballot_sync(kFull, imp & 4u), b3 = __ballot_sync(kFull, imp & 8u);
        // improving lanes lower the word's pending minimum themselves
        if (imp) atomicMin(a.wmin + (w >> 5), best);
        if (hl == 0) {
          const unsigned sh = 16u * half;
          const unsigned long long mask =
              (unsigned long long)((b0 >> sh) & 0xFFFFu) |
              ((unsigned long long)((b1 >> sh) & 0xFFFFu) << 16) |
              ((unsigned long long)((b2 >> sh) & 0xFFFFu) << 32) |
              ((unsigned long long)((b3 >> sh) & 0xFFFFu) << 48);
          if (mask) {
            atomicOr(a.front + w, mask);
            mark_pending<MS_SSSP>(a, w);
          }
        }
      }
      issue(st + kMsRing);
    }
  }
}

// masks with at most this many sources relax lane-per-edge instead
constexpr int kSparseMask = 4;
// BFS groups of small vertices: edges per lane per step (8 spills at 64
// registers)
constexpr int kMsGroupPer = 4;

template <int OP, int ESZ>
__device__ __forceinline__ void ms_edge(const MsArgs &a, uint32_t u, uint32_t w,
                                        uint32_t wt, unsigned long long f, uint32_t lvl1) {
  if (OP == MS_BFS) ms_bfs_edge(a, w, f, lvl1);
  else ms_sssp_edge(a, u, w, wt, f);
}

template <int OP, int ESZ>
__device__ __forceinline__ void ms_chunk(const MsArgs &a, uint32_t ring, const WorkItem &it,
                                         unsigned long long f, uint32_t lvl1) {
  if (OP == MS_SSSP && __popcll(f) > kSparseMask) {
    ms_sssp_item<ESZ>(a, ring, it.v, it.eaddr, it.cnt, f);
    return;
  }
  constexpr int PER = 16 / ESZ;
  const unsigned lane = lane_id();
  const uintptr_t start = it.eaddr;
  const uintptr_t end = start + (uintptr_t)it.cnt * ESZ;
  if (OP == MS_BFS) {
    // two 16-byte loads per lane per step, all their edges probed together
    for (uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane; p < end; p += 1024u) {
      uint32_t w[2 * PER];
      unsigned long long fm[2 * PER];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const uintptr_t ph = p + 512u * h;
        const uint4 q = ph < end ? ld_nc_v4(ph) : make_uint4(0, 0, 0, 0);
        const uint32_t e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < PER; j++) {
          const uintptr_t ea = ph + (uintptr_t)ESZ * j;
          w[h * PER + j] = ESZ == 4 ? edge_dst(e[j], a.wshift) : e[2 * j];
          fm[h * PER + j] = ea >= start && ea < end ? f : 0ull;
        }
      }
      ms_bfs_edges<2 * PER>(a, w, fm, lvl1);
    }
    return;
  }
  for (uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane; p < end; p += 512u) {
    const uint4 q = ld_nc_v4(p);
    const uint32_t e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int j = 0; j < PER; j++) {
      const uintptr_t ea = p + (uintptr_t)ESZ * j;
      if (ea >= start && ea < end)
        ms_edge<OP, ESZ>(a, it.v, ESZ == 4 ? edge_dst(e[j], a.wshift) : e[2 * j],
                         ESZ == 4 ? edge_wt(e[j], a.wshift, a.wbase) : e[2 * j + 1], f, lvl1);
    }
  }
}

// Up to gsize queued vertices per warp (q, qmask: the small or the medium
// bucket's queue): lanes share their concatenated adjacency, so a vertex
// gets about 32 / gsize lanes.  GS = 32 fixes gsize at compile time (the
// two-bucket kernels); GS = 0 takes it from the argument.
template <int OP, int ESZ, int GS>
__device__ __forceinline__ void ms_group(const MsArgs &a, uint32_t ring, const WorkItem *q,
                                         const unsigned long long *qmask, unsigned long long first,
                                         unsigned long long n_items, unsigned gsize,
                                         uint32_t lvl1) {
  const unsigned lane = lane_id();
  const unsigned long long idx = first + lane;
  WorkItem it{0, 0, 0};
  unsigned long long f = 0;
  if ((GS == 32 || lane < gsize) && idx < n_items) {
    it = q[idx];
    f = qmask[idx];
  }
  if (OP == MS_SSSP) {
    // items with dense masks: one at a time, lanes = sources
    unsigned dense = __ballot_sync(kFull, __popcll(f) > kSparseMask);
    while (dense) {
      const int i = __ffs(dense) - 1;
      dense &= dense - 1;
      ms_sssp_item<ESZ>(a, ring, __shfl_sync(kFull, it.v, i), (uintptr_t)shfl64(it.eaddr, i),
                   __shfl_sync(kFull, it.cnt, i), shfl64(f, i));
    }
    if (__popcll(f) > kSparseMask) {
      it.cnt = 0;
      f = 0;
    }
  }
  const unsigned incl = warp_incl_scan<unsigned>(it.cnt);
  const unsigned excl = incl - it.cnt;
  const unsigned total = __shfl_sync(kFull, incl, 31);
  if (OP == MS_BFS) {
    // kMsGroupPer edges per lane per step, probed together
    for (unsigned k = 0; k < total; k += 32u * kMsGroupPer) {
      uint32_t w[kMsGroupPer];
      unsigned long long fm[kMsGroupPer];
#pragma unroll
      for (int h = 0; h < kMsGroupPer; h++) {
        const unsigned t = k + 32u * h + lane;
        const int o = warp_owner(excl, t);
        const unsigned long long ea = shfl64(it.eaddr, o);
        const unsigned oex = __shfl_sync(kFull, excl, o);
        const unsigned long long of = shfl64(f, o);
        w[h] = 0;
        fm[h] = 0;
        if (t < total) {
          const uintptr_t addr = (uintptr_t)ea + (uintptr_t)(t - oex) * ESZ;
          w[h] = ESZ == 4 ? edge_dst(ld_nc_u32(addr), a.wshift) : ld_nc_u2(addr).x;
          fm[h] = of;
        }
      }
      ms_bfs_edges<kMsGroupPer>(a, w, fm, lvl1);
    }
    return;
  }
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
        ms_edge<OP, ESZ>(a, ou, edge_dst(r, a.wshift), edge_wt(r, a.wshift, a.wbase), of, lvl1);
      } else {
        const uint2 e = ld_nc_u2(addr);
        ms_edge<OP, ESZ>(a, ou, e.x, e.y, of, lvl1);
      }
    }
  }
}

// GS = 32: two degree buckets (small groups of 32 vertices per warp, chunks
// above), the launch for the default and most tuned configurations; GS = 0:
// three buckets with the groups' sizes from the arguments.
template <int OP, int ESZ, int THREADS, int GS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) ms_kernel(MsArgs a) {
  // dynamic shared memory: SSSP's per-warp rings, then the block table
  extern __shared__ uint4 s_dyn[];
  constexpr uint32_t ring_words = OP == MS_SSSP ? THREADS / 32 * kMsRing * 32 : 0;
  uint32_t *s_vb = reinterpret_cast<uint32_t *>(s_dyn + ring_words);
  const uint32_t ring = (uint32_t)__cvta_generic_to_shared(s_dyn) +
                        ((threadIdx.x >> 5) * kMsRing * 32u + (threadIdx.x & 31u)) * 16u;
  const bool smem_tab = a.nblk <= kSmemBlocks;
  if (smem_tab)
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];
  __syncthreads();
  const uint32_t *vb = smem_tab ? s_vb : a.blk_vb;
  MsCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  uint32_t thr = OP == MS_SSSP ? (uint32_t)min(1ull + a.delta, 0xFFFFFFFFull) : 0xFFFFFFFFu;
  uint32_t width = a.delta;
  unsigned iter = 0, level = 1;  // BFS level of the vertices being expanded
  if (a.resume) {
    iter = a.r_iter;
    level = a.r_level;
    thr = a.r_thr;
    width = a.r_width;
  }
  bool yielded = false;
  for (;; ++iter) {
    // live groups return here, between iterations: every block has passed
    // the previous iteration's last barrier, and the counter slot of this
    // iteration was cleared during the previous one, so a later launch
    // resumes exactly here
    if (a.yield_at && iter >= a.yield_at) {
      if (leader) {
        c->y_iter = iter;
        c->y_level = level;
        c->y_thr = thr;
        c->y_width = width;
      }
      yielded = true;
      break;
    }
    if (iter >= a.max_iters || (OP == MS_BFS && level > kMaxBfsLevel)) {
      if (leader) atomicCAS(&c->err, 0u, OP == MS_BFS && level > kMaxBfsLevel ? kDevErrDepth : kDevErrIters);
      break;
    }
    const unsigned slot = iter % 3, nslot = (iter + 1) % 3;
    if (leader) {
      c->cnt_small[nslot] = 0;
      c->cnt_big[nslot] = 0;
      c->cnt_mid[nslot] = 0;
      c->remaining[nslot] = 0;
      c->wc[nslot] = 0;
      c->minkept[nslot] = 0xFFFFFFFFu;
    }
    // ---------------------------------------------------------- compaction
    unsigned long long my_edges = 0, my_hbm = 0, my_link = 0, my_pairs = 0, my_keep = 0;
    uint32_t my_min = 0xFFFFFFFFu;
    for (unsigned g = gwarp; g < a.ngroups; g += nwarps) {
      const unsigned wbase = g * 32u;
      const uint32_t word = ldcg(a.bm + wbase + lane);
      unsigned nz = __ballot_sync(kFull, word != 0);
      if (OP == MS_SSSP) {
        const uint32_t wm = word ? ldcg(a.wmin + wbase + lane) : 0xFFFFFFFFu;
        if (word != 0 && wm >= thr) {
          my_keep += __popc(word);
          my_min = min(my_min, wm);
        }
        nz = __ballot_sync(kFull, word != 0 && wm < thr);
      }
      while (nz) {
        const int j = __ffs(nz) - 1;
        nz &= nz - 1;
        const uint32_t wd = __shfl_sync(kFull, word, j);
        const uint32_t v = (wbase + j) * 32u + lane;
        const bool act = (wd >> lane) & 1u;
        unsigned long long take = 0, keep = 0;
        uint32_t kmin = 0xFFFFFFFFu;
        if (act) {
          const unsigned long long f = ldcg(a.front + v);
          if (OP == MS_BFS) {
            take = f;
          } else {
            // the pending sources' distances, eight loads in flight
            const uint32_t *dv = a.dist + (size_t)v * kMsWidth;
            unsigned long long r = f;
            while (r) {
              int s[8];
              uint32_t d[8];
#pragma unroll
              for (int k = 0; k < 8; k++) {
                s[k] = r ? __ffsll((long long)r) - 1 : -1;
                r &= r - 1;
              }
#pragma unroll
              for (int k = 0; k < 8; k++) d[k] = s[k] >= 0 ? ldcg(dv + row_pos((uint32_t)s[k])) : 0u;
#pragma unroll
              for (int k = 0; k < 8; k++) {
                if (s[k] < 0) continue;
                if (d[k] < thr) take |= 1ull << s[k];
                else kmin = min(kmin, d[k]);
              }
            }
            keep = f & ~take;
          }
          a.front[v] = keep;
        }
        const unsigned km = __ballot_sync(kFull, keep != 0);
        if (OP == MS_SSSP) {
          const uint32_t wk = warp_min(kmin);
          my_min = min(my_min, wk);
          if (lane == 0) {
            my_keep += __popc(km);
            a.wmin[wbase + j] = wk;
          }
        }
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
        const bool mid = GS == 0 && take && deg >= a.small_deg && deg < a.mid_deg;
        const bool big = take && deg >= (GS == 0 ? max(a.small_deg, a.mid_deg) : a.small_deg);
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
        const unsigned mm = GS == 0 && a.mid_deg > a.small_deg ? __ballot_sync(kFull, mid) : 0u;
        if (mm) {
          const int ldr = __ffs(mm) - 1;
          unsigned long long base = 0;
          if (lane == (unsigned)ldr)
            base = atomicAdd(&c->cnt_mid[slot], (unsigned long long)__popc(mm));
          base = shfl64(base, ldr);
          const unsigned long long pos = base + __popc(mm & lanemask_lt());
          if (mid) {
            if (pos < a.cap_s) {
              a.qm[pos] = WorkItem{eaddr, v, deg};
              a.qmm[pos] = take;
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
    my_edges = warp_sum(my_edges);
    my_hbm = warp_sum(my_hbm);
    my_link = warp_sum(my_link);
    my_pairs = warp_sum(my_pairs);
    if (lane == 0 && my_edges + my_pairs) {
      atomicAdd(&c->edges, my_edges);
      atomicAdd(&c->hbm_bytes, my_hbm);
      atomicAdd(&c->link_bytes, my_link);
      atomicAdd(&c->pairs, my_pairs);
    }
    if (OP == MS_SSSP) {
      my_keep = warp_sum(my_keep);
      my_min = warp_min(my_min);
      if (lane == 0) {
        if (my_keep) atomicAdd(&c->remaining[slot], my_keep);
        if (my_min != 0xFFFFFFFFu) atomicMin(&c->minkept[slot], my_min);
      }
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
    const unsigned long long ns = ldcg(&c->cnt_small[slot]);
    const unsigned long long nb = ldcg(&c->cnt_big[slot]);
    const unsigned long long nm = GS == 0 ? ldcg(&c->cnt_mid[slot]) : 0ull;
    if (ns + nb + nm == 0) {
      if (OP == MS_BFS) break;
      if (ldcg(&c->remaining[slot]) == 0) break;
      width = (uint32_t)min((unsigned long long)width * a.growth, 0xFFFFFFFFull);
      thr = (uint32_t)min((unsigned long long)ldcg(&c->minkept[slot]) + width, 0xFFFFFFFFull);
      continue;
    }
    // ----------------------------------------------------------- expansion
    const uint32_t lvl1 = level + 1;
    const unsigned gsmall = GS ? GS : a.gsmall;
    const unsigned long long nmt = GS ? 0ull : (nm + a.gmid - 1) / a.gmid;
    const unsigned long long ntask = nb + nmt + (ns + gsmall - 1) / gsmall;
    for (unsigned long long t = gwarp; t < ntask;) {
      if (t < nb) {
        ms_chunk<OP, ESZ>(a, ring, a.qb[t], a.qbm[t], lvl1);
      } else {
        // one inlined copy of the group code serves both grouped buckets
        const bool md = GS == 0 && t < nb + nmt;
        ms_group<OP, ESZ, GS>(a, ring, md ? a.qm : a.qs, md ? a.qmm : a.qsm,
                              md ? (t - nb) * a.gmid : (t - nb - nmt) * gsmall, md ? nm : ns,
                              md ? a.gmid : gsmall, lvl1);
      }
      unsigned long long nt = 0;
      if (lane == 0) nt = nwarps + atomicAdd(&c->wc[slot], 1ull);
      t = shfl64(nt, 0);
    }
    level++;
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
  }
  if (leader) {
    c->iters = iter;
    c->yielded = yielded ? 1u : 0u;
  }
}

template <int OP>
__global__ void ms_init(MsArgs a, uint32_t nw_alloc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t v = tid; v < a.nv; v += stride) {
    a.front[v] = 0;
    if (OP == MS_BFS) a.visit[v] = 0;
  }
  // per-source rows as one flat array of 16-byte words, consecutive threads
  // on consecutive words
  if (OP == MS_BFS) {
    uint4 *rows = reinterpret_cast<uint4 *>(a.lvl);
    for (uint64_t i = tid; i < a.nv * (kMsWidth / 16); i += stride) rows[i] = make_uint4(0, 0, 0, 0);
  } else {
    uint4 *rows = reinterpret_cast<uint4 *>(a.dist);
    const uint32_t inf = a.nv + 1u;
    for (uint64_t i = tid; i < a.nv * (kMsWidth / 4); i += stride) rows[i] = make_uint4(inf, inf, inf, inf);
  }
  for (uint64_t w = tid; w < nw_alloc; w += stride) {
    a.bm[w] = 0;
    if (OP == MS_SSSP) a.wmin[w] = 0xFFFFFFFFu;
  }
  if (tid == 0) {
    memset(a.ctrl, 0, sizeof(MsCtrl));
    for (int s = 0; s < 3; s++) a.ctrl->minkept[s] = 0xFFFFFFFFu;
  }
}

// Sources go in after the reset (same stream, next launch): duplicates in a
// group are distinct bits of the same vertex.
template <int OP>
__global__ void ms_seed(MsArgs a) {
  const uint32_t s = threadIdx.x;
  if (s >= a.sources[0]) return;
  const uint32_t v = a.sources[1 + s];
  atomicOr(a.front + v, 1ull << s);
  atomicOr(a.bm + (v >> 5), 1u << (v & 31u));
  if (OP == MS_BFS) {
    atomicOr(a.visit + v, 1ull << s);
    a.lvl[(size_t)v * kMsWidth + s] = 1;
  } else {
    a.dist[(size_t)v * kMsWidth + row_pos(s)] = 1;
    atomicMin(a.wmin + (v >> 5), 1u);
  }
}

__device__ __forceinline__ unsigned long long value_hash(uint32_t v, uint32_t val) {
  unsigned long long x = ((unsigned long long)v << 32) | val;
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

constexpr uint32_t kExtractThreads = 256;  // ms_extract's block: 32 vertices x 64 sources per tile
constexpr uint32_t kExtractPer = 32 * kMsWidth / kExtractThreads;

// Per-source values in the single-source encoding: optional k x nv output
// (rows per source) and a checksum per source (sum of value_hash(v, val)).

template <int OP>
__global__ void __launch_bounds__(kExtractThreads) ms_extract(MsArgs a, uint32_t *out,
                                                             unsigned long long *sums) {
  __shared__ unsigned long long s_sum[kMsWidth];
  __shared__ uint32_t tile[32][kMsWidth + 1];
  const uint32_t k = a.sources[0];
  for (uint32_t i = threadIdx.x; i < kMsWidth; i += blockDim.x) s_sum[i] = 0;
  // a warp always reads sources warp + 8j of a tile (j < kExtractPer), one
  // vertex per lane: the hashes add up in registers across tiles
  unsigned long long acc[kExtractPer];
#pragma unroll
  for (uint32_t j = 0; j < kExtractPer; j++) acc[j] = 0;
  __syncthreads();
  const uint32_t inf = a.nv + 1u;
  for (uint64_t base = (uint64_t)blockIdx.x * 32; base < a.nv; base += (uint64_t)gridDim.x * 32) {
    for (uint32_t i = threadIdx.x; i < 32 * kMsWidth; i += kExtractThreads) {
      const uint32_t dv = i / kMsWidth, s = i % kMsWidth;
      const uint64_t v = base + dv;
      uint32_t val = inf;
      if (v < a.nv) {
        if (OP == MS_BFS) {
          const uint8_t l = a.lvl[v * kMsWidth + s];
          val = l ? l : inf;
        } else {
          val = a.dist[v * kMsWidth + row_pos(s)];
        }
      }
      tile[dv][s] = val;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t j = 0; j < kExtractPer; j++) {
      const uint32_t i = threadIdx.x + j * kExtractThreads;
      const uint32_t s = i / 32, dv = i % 32;
      const uint64_t v = base + dv;
      if (s < k && v < a.nv) {
        const uint32_t val = tile[dv][s];
        if (out) out[(uint64_t)s * a.nv + v] = val;
        acc[j] += value_hash((uint32_t)v, val);
      }
    }
    __syncthreads();
  }
  if (!sums) return;
#pragma unroll
  for (uint32_t j = 0; j < kExtractPer; j++) {
    const unsigned long long t = warp_sum(acc[j]);
    if (lane_id() == 0 && t) atomicAdd(&s_sum[(threadIdx.x + j * kExtractThreads) / 32], t);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < k; i += blockDim.x)
    if (s_sum[i]) atomicAdd(sums + i, s_sum[i]);
}

// Checksums only (no output rows): rows are read as they lie, 16 lanes per
// row, and each lane keeps the sums of its four sources in registers (SSSP:
// one 16-byte word = sources l, l+16, l+32, l+48; BFS: one 4-byte word =
// level bytes of sources 4l..4l+3).
template <int OP>
__global__ void __launch_bounds__(kExtractThreads) ms_checksum(MsArgs a, unsigned long long *sums) {
  __shared__ unsigned long long s_sum[kMsWidth];
  const uint32_t k = a.sources[0];
  for (uint32_t i = threadIdx.x; i < kMsWidth; i += blockDim.x) s_sum[i] = 0;
  __syncthreads();
  const uint32_t l = threadIdx.x & 15u, inf = a.nv + 1u;
  uint32_t src[4];
#pragma unroll
  for (int i = 0; i < 4; i++) src[i] = OP == MS_BFS ? 4u * l + i : l + 16u * i;
  unsigned long long acc[4] = {0, 0, 0, 0};
  const uint64_t rows_per = kExtractThreads / 16;
  for (uint64_t v = (uint64_t)blockIdx.x * rows_per + threadIdx.x / 16; v < a.nv;
       v += (uint64_t)gridDim.x * rows_per) {
    uint32_t val[4];
    if (OP == MS_BFS) {
      const uint32_t b = __ldcs(reinterpret_cast<const uint32_t *>(a.lvl + v * kMsWidth) + l);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t x = (b >> (8 * i)) & 0xFFu;
        val[i] = x ? x : inf;
      }
    } else {
      const uint4 d = __ldcs(reinterpret_cast<const uint4 *>(a.dist + v * kMsWidth) + l);
      val[0] = d.x;
      val[1] = d.y;
      val[2] = d.z;
      val[3] = d.w;
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (src[i] < k) acc[i] += value_hash((uint32_t)v, val[i]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const unsigned long long t = acc[i] + __shfl_xor_sync(kFull, acc[i], 16);
    if ((threadIdx.x & 31u) < 16u && t) atomicAdd(&s_sum[src[i]], t);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < k; i += blockDim.x)
    if (s_sum[i]) atomicAdd(sums + i, s_sum[i]);
}

// ------------------------------------------------------- live groups --
// Continuous batching (the server): one group per algorithm stays on the
// device between launches; arrivals take free mask bits and sources whose
// pending set is empty retire, both between launches.  A source that joins
// a running group keeps the single-source encoding relative to its start:
//   BFS  its source vertex gets the group's current level byte L (the level
//        expanded next), so its value at v is lvl[v][s] - (L - 1);
//   SSSP its source vertex gets the current window's lower end b, so its
//        value at v is dist[v][s] - (b - 1); its column starts at nv + b,
//        the single-source "unreached" nv + 1 shifted the same way, so a
//        relaxation stores only what the single-source run would store
//        (distances below nv + 1).  The shared window then treats it as a
//        source that started at distance b, the other sources' scale.
// A group that has always started its sources at L = 1 / b = 1 is the
// plain batched group.

// OR of every vertex's pending-source mask: the sources still running.
__global__ void ms_alive(const unsigned long long *front, uint32_t nv, unsigned long long *out) {
  unsigned long long m = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x)
    m |= __ldcs(front + v);
  m = warp_or(m);
  if (lane_id() == 0 && m) atomicOr(out, m);
}

// Expands the low 4 bits of n into a byte mask (bit i -> byte i).
__device__ __forceinline__ uint32_t byte_mask4(uint32_t n) {
  return ((n & 1u) ? 0xFFu : 0u) | ((n & 2u) ? 0xFF00u : 0u) | ((n & 4u) ? 0xFF0000u : 0u) |
         ((n & 8u) ? 0xFF000000u : 0u);
}

// Columns of the joining sources jm back to "unreached", 16 bytes of a row
// per thread: BFS clears their visit bits and level bytes, SSSP writes each
// source's shifted unreached value unreached[s].  Pending masks of these
// bits are already empty (retired or never used).
template <int OP>
__global__ void ms_live_reset(MsArgs a, unsigned long long jm, const uint32_t *unreached) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (OP == MS_BFS) {
    for (uint64_t v = tid; v < a.nv; v += stride) a.visit[v] &= ~jm;
    uint4 *rows = reinterpret_cast<uint4 *>(a.lvl);
    for (uint64_t i = tid; i < (uint64_t)a.nv * 4u; i += stride) {
      const uint32_t q = (uint32_t)(i & 3u);  // bytes 16q .. 16q+15: sources 16q ..
      const uint32_t bits = (uint32_t)(jm >> (16u * q)) & 0xFFFFu;
      if (!bits) continue;
      uint4 w = rows[i];
      w.x &= ~byte_mask4(bits);
      w.y &= ~byte_mask4(bits >> 4);
      w.z &= ~byte_mask4(bits >> 8);
      w.w &= ~byte_mask4(bits >> 12);
      rows[i] = w;
    }
  } else {
    uint4 *rows = reinterpret_cast<uint4 *>(a.dist);
    for (uint64_t i = tid; i < (uint64_t)a.nv * 16u; i += stride) {
      const uint32_t p = (uint32_t)(i & 15u);  // piece p: sources p, p+16, p+32, p+48
      const uint32_t sel = (uint32_t)((jm >> p) & 1ull) | (uint32_t)((jm >> (p + 15u)) & 2ull) |
                           (uint32_t)((jm >> (p + 30u)) & 4ull) | (uint32_t)((jm >> (p + 45u)) & 8ull);
      if (!sel) continue;
      uint4 w = rows[i];
      if (sel & 1u) w.x = __ldg(unreached + p);
      if (sel & 2u) w.y = __ldg(unreached + p + 16u);
      if (sel & 4u) w.z = __ldg(unreached + p + 32u);
      if (sel & 8u) w.w = __ldg(unreached + p + 48u);
      rows[i] = w;
    }
  }
}

// k joining sources: bit bits[t] starts at vertex srcs[t] with value
// vals[t] (BFS level byte, SSSP distance).
template <int OP>
__global__ void ms_live_seed(MsArgs a, uint32_t k, const uint32_t *bits, const uint32_t *srcs,
                             const uint32_t *vals) {
  const uint32_t t = threadIdx.x;
  if (t >= k) return;
  const uint32_t s = bits[t], v = srcs[t], val = vals[t];
  atomicOr(a.front + v, 1ull << s);
  atomicOr(a.bm + (v >> 5), 1u << (v & 31u));
  if (OP == MS_BFS) {
    atomicOr(a.visit + v, 1ull << s);
    a.lvl[(size_t)v * kMsWidth + s] = (uint8_t)val;
  } else {
    a.dist[(size_t)v * kMsWidth + row_pos(s)] = val;
    atomicMin(a.wmin + (v >> 5), val);
  }
}

// Value of source s at a stored entry, in the single-source encoding, for a
// source started at base b (BFS level byte / SSSP distance of its vertex).
template <int OP>
__device__ __forceinline__ uint32_t live_value(uint32_t raw, uint32_t b, uint32_t nv) {
  if (OP == MS_BFS) return raw ? raw - (b - 1u) : nv + 1u;
  return raw >= nv + b ? nv + 1u : raw - (b - 1u);
}

// Checksums of the finishing sources fin (rows read as they lie, only the
// pieces holding a finishing source; see ms_checksum).
template <int OP>
__global__ void __launch_bounds__(kExtractThreads) ms_live_sums(MsArgs a, unsigned long long fin,
                                                                const uint32_t *base,
                                                                unsigned long long *sums) {
  __shared__ unsigned long long s_sum[kMsWidth];
  for (uint32_t i = threadIdx.x; i < kMsWidth; i += blockDim.x) s_sum[i] = 0;
  __syncthreads();
  const uint32_t l = threadIdx.x & 15u;
  uint32_t src[4], b[4];
  bool want[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    src[i] = OP == MS_BFS ? 4u * l + i : l + 16u * i;
    want[i] = (fin >> src[i]) & 1ull;
    b[i] = want[i] ? __ldg(base + src[i]) : 1u;
  }
  const bool any = want[0] || want[1] || want[2] || want[3];
  unsigned long long acc[4] = {0, 0, 0, 0};
  const uint64_t rows_per = kExtractThreads / 16;
  for (uint64_t v = (uint64_t)blockIdx.x * rows_per + threadIdx.x / 16; any && v < a.nv;
       v += (uint64_t)gridDim.x * rows_per) {
    uint32_t raw[4];
    if (OP == MS_BFS) {
      const uint32_t w = __ldcs(reinterpret_cast<const uint32_t *>(a.lvl + v * kMsWidth) + l);
#pragma unroll
      for (int i = 0; i < 4; i++) raw[i] = (w >> (8 * i)) & 0xFFu;
    } else {
      const uint4 d = __ldcs(reinterpret_cast<const uint4 *>(a.dist + v * kMsWidth) + l);
      raw[0] = d.x;
      raw[1] = d.y;
      raw[2] = d.z;
      raw[3] = d.w;
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (want[i]) acc[i] += value_hash((uint32_t)v, live_value<OP>(raw[i], b[i], a.nv));
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const unsigned long long t = acc[i] + __shfl_xor_sync(kFull, acc[i], 16);
    if ((threadIdx.x & 31u) < 16u && t) atomicAdd(&s_sum[src[i]], t);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < kMsWidth; i += blockDim.x)
    if (((fin >> i) & 1ull) && s_sum[i]) atomicAdd(sums + i, s_sum[i]);
}

// Values of one source (bit s, base b) into out[nv].
template <int OP>
__global__ void ms_live_column(MsArgs a, uint32_t s, uint32_t b, uint32_t *out) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < a.nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t raw = OP == MS_BFS ? (uint32_t)a.lvl[v * kMsWidth + s]
                                      : a.dist[v * kMsWidth + row_pos(s)];
    out[v] = live_value<OP>(raw, b, a.nv);
  }
}

// ------------------------------------------------------------------ host --

// Launch configuration of the batch kernel, per degree bucket:
//   [1, small)    groups of gsmall vertices per warp (about 32 / gsmall
//                 lanes per vertex, load-balanced over their edges);
//   [small, mid)  groups of gmid vertices per warp (empty when mid <= small);
//   [mid, ...)    chunks of `chunk` edges, one warp each;
// and the threads per CTA of the one persistent launch.
struct MsConfig {
  uint32_t small, chunk, threads, mid, gsmall, gmid;
  bool operator<(const MsConfig &o) const {
    return std::tie(small, chunk, threads, mid, gsmall, gmid) <
           std::tie(o.small, o.chunk, o.threads, o.mid, o.gsmall, o.gmid);
  }
};

constexpr MsConfig kMsDefault{64, 256, 512, 64, 32, 4};
constexpr uint32_t kMsMinSmall = 16, kMsMinChunk = 128;
// Grouped buckets stop at 2^20 edges per vertex, so a warp's group (at most
// 32 lists) counts its edges in 32 bits.
constexpr uint32_t kMsMaxGroupedDeg = 1u << 20;

// A captured launch sequence holds its kernel arguments by value, so the key
// covers every argument that can differ between calls on one batch state.
struct GraphKey {
  int op, esz, threads;
  bool out;
  uint32_t small, chunk, delta, growth, mid, gsmall, gmid;
  unsigned long long timeout_ns;
  bool operator<(const GraphKey &o) const {
    return std::tie(op, esz, threads, out, small, chunk, delta, growth, mid, gsmall, gmid,
                    timeout_ns) <
           std::tie(o.op, o.esz, o.threads, o.out, o.small, o.chunk, o.delta, o.growth, o.mid,
                    o.gsmall, o.gmid, o.timeout_ns);
  }
};

// THV_BATCH_DIRECT=1 launches every group directly instead of replaying a
// captured graph (kernel profilers list cooperative kernels launched from a
// graph poorly); results are the same either way.
static bool batch_capture_allowed() {
  const char *e = getenv("THV_BATCH_DIRECT");
  return !(e && e[0] == '1');
}

struct BatchExtra {
  std::map<GraphKey, cudaGraphExec_t> graphs;
  bool capture_ok = batch_capture_allowed();
};

static std::map<BatchState *, BatchExtra> g_extra;  // graphs per batch state
static std::mutex g_tune_mu;
static std::map<std::string, MsConfig> g_tune;     // in-process tuner cache

static void free_state(BatchState *&b) {
  if (!b) return;
  auto it = g_extra.find(b);
  if (it != g_extra.end()) {
    for (auto &kv : it->second.graphs) cudaGraphExecDestroy(kv.second);
    g_extra.erase(it);
  }
  dev_free(b->d_visit);
  dev_free(b->d_front);
  dev_free(b->d_lvl);
  dev_free(b->d_dist);
  dev_free(b->d_bm);
  dev_free(b->d_wmin);
  dev_free(b->d_qs);
  dev_free(b->d_qb);
  dev_free(b->d_qsm);
  dev_free(b->d_qbm);
  dev_free(b->d_qm);
  dev_free(b->d_qmm);
  dev_free(b->d_ctrl);
  pinned_free(b->h_ctrl);
  dev_free(b->d_sources);
  pinned_free(b->h_sources);
  dev_free(b->d_out);
  dev_free(b->d_sums);
  pinned_free(b->h_sums);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
  b = nullptr;
}

void batch_free(thv_graph *g) {
  free_state(g->bs_keep[0]);
  free_state(g->bs_keep[1]);
  g->bs = nullptr;
}

// Queues are sized for the smallest bucket boundary and chunk any
// configuration may use, so tuning never reallocates.  BFS and SSSP keep
// separate states, so alternating between them (served groups) does not
// reallocate either.
static thv_status fill_batch_state(thv_graph *g, BatchState *b, bool sssp, bool want_out);

static thv_status ensure_batch_state(thv_graph *g, bool sssp, bool want_out) {
  BatchState *&b = g->bs_keep[sssp ? 1 : 0];
  g->bs = nullptr;
  if (b && b->valid && (!want_out || b->d_out)) {
    g->bs = b;
    return THV_OK;
  }
  free_state(b);
  b = new BatchState();
  g->bs = b;
  return fill_batch_state(g, b, sssp, want_out);
}

// Allocates every buffer of b (b->valid once all succeeded).
static thv_status fill_batch_state(thv_graph *g, BatchState *b, bool sssp, bool want_out) {
  b->nv = g->nv;
  b->sssp = sssp;
  const uint64_t nw = (g->nv + 31) / 32;
  b->ngroups = (uint32_t)((nw + 31) / 32);
  const uint64_t nw_alloc = (uint64_t)b->ngroups * 32;
  b->cap_s = g->nv + 32;
  b->cap_b = g->ne / kMsMinChunk + g->ne / kMsMinSmall + 64;
  THV_TRY(dev_alloc((void **)&b->d_front, g->nv * 8 + 64, "batch frontier masks"));
  if (sssp) {
    THV_TRY(dev_alloc((void **)&b->d_dist, g->nv * kMsWidth * 4 + 64, "batch distances"));
  } else {
    THV_TRY(dev_alloc((void **)&b->d_visit, g->nv * 8 + 64, "batch visit masks"));
    THV_TRY(dev_alloc((void **)&b->d_lvl, g->nv * kMsWidth + 64, "batch levels"));
  }
  THV_TRY(dev_alloc((void **)&b->d_bm, nw_alloc * 4, "batch pending bitmap"));
  THV_TRY(dev_alloc((void **)&b->d_wmin, nw_alloc * 4, "batch pending minima"));
  THV_TRY(dev_alloc((void **)&b->d_qs, b->cap_s * sizeof(WorkItem), "batch queue"));
  THV_TRY(dev_alloc((void **)&b->d_qsm, b->cap_s * 8, "batch queue masks"));
  THV_TRY(dev_alloc((void **)&b->d_qm, b->cap_s * sizeof(WorkItem), "batch medium queue"));
  THV_TRY(dev_alloc((void **)&b->d_qmm, b->cap_s * 8, "batch medium queue masks"));
  THV_TRY(dev_alloc((void **)&b->d_qb, b->cap_b * sizeof(WorkItem), "batch chunk queue"));
  THV_TRY(dev_alloc((void **)&b->d_qbm, b->cap_b * 8, "batch chunk masks"));
  THV_TRY(dev_alloc((void **)&b->d_ctrl, sizeof(MsCtrl), "batch control"));
  THV_TRY(pinned_alloc((void **)&b->h_ctrl, sizeof(MsCtrl), "batch control"));
  THV_TRY(dev_alloc((void **)&b->d_sources, (kMsWidth + 1) * 4, "batch sources"));
  THV_TRY(pinned_alloc((void **)&b->h_sources, (kMsWidth + 1) * 4, "batch sources"));
  THV_TRY(dev_alloc((void **)&b->d_sums, kMsWidth * 8, "batch checksums"));
  THV_TRY(pinned_alloc((void **)&b->h_sums, kMsWidth * 8, "batch checksums"));
  if (want_out) THV_TRY(dev_alloc((void **)&b->d_out, (uint64_t)kMsWidth * g->nv * 4 + 64, "batch output"));
  THV_CUDA(cudaEventCreate(&b->ev0));
  THV_CUDA(cudaEventCreate(&b->ev1));
  b->valid = true;
  return THV_OK;
}

// The whole group -- sources up, reset, seed, persistent traversal,
// extraction, status down -- enqueued on `st` (captured into a graph once).
// The two-bucket kernel serves configurations without a medium bucket and
// with 32 small vertices per warp.
static bool two_buckets(const MsArgs &a) { return a.gsmall == 32 && a.mid_deg <= a.small_deg; }

template <int OP, int ESZ, int THREADS>
static thv_status enqueue_group(thv_graph *g, MsArgs &a, cudaStream_t st, bool want_out) {
  BatchState *b = g->bs;
  auto kern = two_buckets(a) ? ms_kernel<OP, ESZ, THREADS, 32> : ms_kernel<OP, ESZ, THREADS, 0>;
  const size_t ring = OP == MS_SSSP ? (size_t)THREADS / 32 * kMsRing * 512 : 0;
  const size_t smem = ring + (g->plan.vbegin.size() <= kSmemBlocks + 1 ? g->plan.vbegin.size() * 4 : 0);
  THV_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int bpsm = 0;
  THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, THREADS, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "batch kernel cannot be resident");
  const int grid = bpsm * g->num_sms;
  const int igrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  THV_CUDA(cudaMemcpyAsync(b->d_sources, b->h_sources, (kMsWidth + 1) * 4, cudaMemcpyHostToDevice, st));
  ms_init<OP><<<igrid, 256, 0, st>>>(a, b->ngroups * 32u);
  ms_seed<OP><<<1, kMsWidth, 0, st>>>(a);
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(THREADS), args, smem, st));
  THV_CUDA(cudaMemsetAsync(b->d_sums, 0, kMsWidth * 8, st));
  const int xgrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 31) / 32)));
  if (want_out)
    ms_extract<OP><<<xgrid, kExtractThreads, 0, st>>>(a, b->d_out, b->d_sums);
  else
    ms_checksum<OP><<<g->num_sms * 8, kExtractThreads, 0, st>>>(a, b->d_sums);
  THV_CUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, sizeof(MsCtrl), cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaMemcpyAsync(b->h_sums, b->d_sums, kMsWidth * 8, cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaGetLastError());
  return THV_OK;
}

template <int OP, int ESZ>
static thv_status enqueue_any(thv_graph *g, MsArgs &a, cudaStream_t st, bool want_out,
                              uint32_t threads) {
  return threads == 256 ? enqueue_group<OP, ESZ, 256>(g, a, st, want_out)
                        : enqueue_group<OP, ESZ, 512>(g, a, st, want_out);
}

static thv_status enqueue(thv_graph *g, bool sssp, MsArgs &a, cudaStream_t st, bool want_out,
                          uint32_t threads) {
  if (sssp) {
    if (!g->weighted) return fail(THV_EINVAL, "SSSP needs edge weights");
    return g->esz == 8 ? enqueue_any<MS_SSSP, 8>(g, a, st, want_out, threads)
                       : enqueue_any<MS_SSSP, 4>(g, a, st, want_out, threads);  // packed
  }
  return g->esz == 8 ? enqueue_any<MS_BFS, 8>(g, a, st, want_out, threads)
                     : enqueue_any<MS_BFS, 4>(g, a, st, want_out, threads);
}

// Runs the group whose sources sit in h_sources; replays a captured CUDA
// graph of the launch sequence when capture works on this stream.
static thv_status run_group(thv_graph *g, bool sssp, MsArgs &a, cudaStream_t st, bool want_out,
                            const MsConfig &cfg, uint32_t &launches) {
  BatchState *b = g->bs;
  BatchExtra &ex = g_extra[b];
  const GraphKey key{sssp ? 1 : 0, (int)g->esz, (int)cfg.threads, want_out, cfg.small, cfg.chunk,
                     a.delta,     a.growth,    a.mid_deg,      a.gsmall, a.gmid, a.timeout_ns};
  auto it = ex.graphs.find(key);
  if (it == ex.graphs.end() && ex.capture_ok) {
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    thv_status s = ok ? enqueue(g, sssp, a, cs, want_out, cfg.threads) : THV_ECUDA;
    if (ok) ok = cudaStreamEndCapture(cs, &graph) == cudaSuccess && s == THV_OK;
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (cs) cudaStreamDestroy(cs);
    cudaGetLastError();
    if (ok) it = ex.graphs.emplace(key, exec).first;
    else ex.capture_ok = false;  // fall back to direct launches from now on
  }
  if (it != ex.graphs.end()) {
    THV_CUDA(cudaGraphLaunch(it->second, st));
    launches += 4;
    return THV_OK;
  }
  THV_TRY(enqueue(g, sssp, a, st, want_out, cfg.threads));
  launches += 4;
  return THV_OK;
}

static unsigned long long host_value_hash(uint32_t v, uint32_t val) {
  unsigned long long x = ((unsigned long long)v << 32) | val;
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static thv_status fallback_single(thv_graph *g, const uint32_t *src, uint32_t k, cudaStream_t st,
                                  const thv_batch_opts *o, uint32_t *const *rows, uint64_t *sums,
                                  thv_stats &acc) {
  std::vector<uint32_t> vals(g->nv);
  for (uint32_t i = 0; i < k; i++) {
    thv_run_opts ro{};
    ro.source = src[i];
    ro.timeout_ms = o ? o->timeout_ms : 0;
    thv_stats st1{};
    THV_TRY(run_minprop(g, THV_ALGO_BFS, &ro, st, &st1));
    uint32_t *dst = rows && rows[i] ? rows[i] : vals.data();
    THV_TRY(minprop_values(g, dst, st));
    if (sums) {
      unsigned long long h = 0;
      for (uint64_t v = 0; v < g->nv; v++) h += host_value_hash((uint32_t)v, dst[v]);
      sums[i] = h;
    }
    acc.device_ms += st1.device_ms;
    acc.iterations += st1.iterations;
    acc.edges_expanded += st1.edges_expanded;
    acc.hbm_edge_bytes += st1.hbm_edge_bytes;
    acc.link_edge_bytes += st1.link_edge_bytes;
  }
  return THV_OK;
}

static std::string tune_key(const thv_graph *g, bool sssp) {
  char buf[160];
  snprintf(buf, sizeof(buf), "%s3 nv=%llu ne=%llu esz=%u resident=%llu blocks=%zu sms=%d",
           sssp ? "sssp" : "bfs", (unsigned long long)g->nv, (unsigned long long)g->ne, g->esz,
           (unsigned long long)g->plan.resident_edge_bytes, g->plan.blocks.size(), g->num_sms);
  return buf;
}

static std::string tune_file() {
  const char *p = getenv("THV_TUNE_CACHE");
  if (p && *p) return p;
  const char *h = getenv("HOME");
  return std::string(h && *h ? h : "/tmp") + "/.cache/thievory_b200_batch_tune.txt";
}

static bool tune_lookup(const std::string &key, MsConfig *cfg) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(key);
  if (it != g_tune.end()) { *cfg = it->second; return true; }
  FILE *f = fopen(tune_file().c_str(), "r");
  if (!f) return false;
  char line[512];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    char *bar = strchr(line, '|');
    if (!bar) continue;
    *bar = 0;
    MsConfig c{};
    if (key == line &&
        sscanf(bar + 1, "%u %u %u %u %u %u", &c.small, &c.chunk, &c.threads, &c.mid, &c.gsmall,
               &c.gmid) == 6 &&
        (c.threads == 256 || c.threads == 512) && c.small >= kMsMinSmall && c.chunk >= kMsMinChunk &&
        c.gsmall >= 1 && c.gsmall <= 32 && c.gmid >= 1 && c.gmid <= 32) {
      *cfg = c;
      found = true;
    }
  }
  fclose(f);
  if (found) g_tune[key] = *cfg;
  return found;
}

static void tune_store(const std::string &key, const MsConfig &c) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = c;
  const std::string path = tune_file();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    std::string dir = path.substr(0, slash);
    (void)!system(("mkdir -p '" + dir + "' 2>/dev/null").c_str());
  }
  FILE *f = fopen(path.c_str(), "a");
  if (!f) return;
  fprintf(f, "%s|%u %u %u %u %u %u\n", key.c_str(), c.small, c.chunk, c.threads, c.mid, c.gsmall,
          c.gmid);
  fclose(f);
}

// Kernel arguments over batch state b (window, growth and tuning left at
// their zero values for the caller to set).
static MsArgs ms_args(thv_graph *g, BatchState *b, uint32_t timeout_ms) {
  MsArgs a{};
  a.off = g->d_off;
  a.blk_vb = g->plan.d_vbegin;
  a.blk_base = g->plan.d_base;
  a.host_base = g->h_edges_dev;
  a.lc = list_cache_of(g->plan);
  a.blk_access = g->plan.d_access;
  a.wshift = g->wshift;
  a.wbase = g->wbase;
  a.visit = b->d_visit;
  a.front = b->d_front;
  a.lvl = b->d_lvl;
  a.dist = b->d_dist;
  a.bm = b->d_bm;
  a.wmin = b->d_wmin;
  a.qs = b->d_qs;
  a.qb = b->d_qb;
  a.qsm = b->d_qsm;
  a.qbm = b->d_qbm;
  a.qm = b->d_qm;
  a.qmm = b->d_qmm;
  a.cap_s = b->cap_s;
  a.cap_b = b->cap_b;
  a.ctrl = b->d_ctrl;
  a.sources = b->d_sources;
  a.timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
  a.nblk = (uint32_t)g->plan.blocks.size();
  a.nv = (uint32_t)g->nv;
  a.ngroups = b->ngroups;
  a.max_iters = (uint32_t)std::min<uint64_t>(g->nv + 2, 0x7FFFFFF0ull) * 2 + 8;
  return a;
}

static void apply_config(MsArgs &a, const MsConfig &c) {
  a.small_deg = std::min(std::max(c.small, kMsMinSmall), kMsMaxGroupedDeg);
  a.chunk = std::max(c.chunk, kMsMinChunk);
  a.mid_deg = std::min(std::max(c.mid, a.small_deg), kMsMaxGroupedDeg);
  a.gsmall = std::min(std::max(c.gsmall, 1u), 32u);
  a.gmid = std::min(std::max(c.gmid, 1u), 32u);
}

thv_status batch_config(thv_graph *g, thv_algo algo, thv_batch_config *out) {
  if (algo != THV_ALGO_BFS && algo != THV_ALGO_SSSP)
    return fail(THV_EINVAL, "batched runs support BFS and SSSP");
  THV_TRY(ensure_plan(g));
  MsConfig c = kMsDefault;
  const bool tuned = tune_lookup(tune_key(g, algo == THV_ALGO_SSSP), &c);
  out->small_degree = c.small;
  out->mid_degree = std::max(c.mid, c.small);
  out->chunk_edges = c.chunk;
  out->threads = c.threads;
  out->small_group = c.gsmall;
  out->mid_group = c.gmid;
  out->tuned = tuned ? 1u : 0u;
  out->pad = 0;
  return THV_OK;
}

thv_status run_batch(thv_graph *g, thv_algo algo, const uint32_t *sources,
                     uint32_t n, const thv_batch_opts *o, uint32_t *out,
                     uint64_t *checksums, thv_stats *stats) {
  std::vector<uint32_t *> rows;
  if (out) {
    rows.resize(n);
    for (uint32_t i = 0; i < n; i++) rows[i] = out + (uint64_t)i * g->nv;
  }
  return run_batch_rows(g, algo, sources, n, o, out ? rows.data() : nullptr, checksums, stats);
}

// As run_batch, with one destination per source (rows[i] may be null; rows
// may be null for checksums only).
thv_status run_batch_rows(thv_graph *g, thv_algo algo, const uint32_t *sources,
                          uint32_t n, const thv_batch_opts *o, uint32_t *const *rows,
                          uint64_t *checksums, thv_stats *stats) {
  bool want_out = false;
  for (uint32_t i = 0; rows && i < n; i++) want_out |= rows[i] != nullptr;
  if (algo != THV_ALGO_BFS && algo != THV_ALGO_SSSP)
    return fail(THV_EINVAL, "batched runs support BFS and SSSP");
  const bool sssp = algo == THV_ALGO_SSSP;
  if (sssp && !g->weighted) return fail(THV_EINVAL, "SSSP needs edge weights");
  if (g->fmt == THV_FMT_CSC) return fail(THV_EINVAL, "batched runs need out-edges (CSR/WCSR)");
  if (g->nv >= 0xFFFFFFFFull) return fail(THV_EUNSUPPORTED, "too many vertices");
  for (uint32_t i = 0; i < n; i++)
    if (sources[i] >= g->nv) return fail(THV_EINVAL, "source %u out of range", sources[i]);
  const uint32_t group = o && o->group ? std::min<uint32_t>(o->group, kMsWidth) : kMsWidth;
  const double t0 = now_ms();
  THV_TRY(ensure_plan(g));
  THV_TRY(ensure_batch_state(g, sssp, want_out));
  BatchState *b = g->bs;
  cudaStream_t st = o && o->stream ? (cudaStream_t)o->stream : g->stream;
  const uint32_t tmo = o && o->timeout_ms ? o->timeout_ms : 60000u;
  MsArgs a = ms_args(g, b, tmo);
  // Wide windows: many sources expand a vertex in the same iteration and
  // share its adjacency read (small windows make each source re-read it).
  // RMAT-26, 256 sources, weights 1..64: width 16 -> 36.6 q/s, 64 -> 74.8,
  // 128 -> 99.3, 256 -> 100.1, unbounded -> 100.1.
  a.delta = o && o->sssp_delta ? o->sssp_delta : kMsDelta;
  a.growth = o && o->sssp_growth ? o->sssp_growth : kMsGrowth;

  thv_stats local{};
  uint32_t launches = 0;
  float dev_ms = 0.f;
  auto set_cfg = [&](const MsConfig &c) { apply_config(a, c); };
  auto one_group = [&](uint32_t first, uint32_t k, const MsConfig &cfg, float *ms_out,
                       bool *deep) -> thv_status {
    set_cfg(cfg);
    b->h_sources[0] = k;
    memcpy(b->h_sources + 1, sources + first, k * 4);
    THV_CUDA(cudaEventRecord(b->ev0, st));
    THV_TRY(run_group(g, sssp, a, st, want_out, cfg, launches));
    THV_CUDA(cudaEventRecord(b->ev1, st));
    for (uint32_t i = 0; want_out && i < k; i++)
      if (rows[first + i])
        THV_CUDA(cudaMemcpyAsync(rows[first + i], b->d_out + (uint64_t)i * g->nv, g->nv * 4,
                                 cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaStreamSynchronize(st));
    cudaEventElapsedTime(ms_out, b->ev0, b->ev1);
    const MsCtrl &hc = *b->h_ctrl;
    *deep = hc.err == kDevErrDepth;
    if (hc.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "grid barrier wait exceeded %u ms", tmo);
    if (hc.err == kDevErrIters) return fail(THV_ETIMEOUT, "iteration cap reached");
    if (hc.err && hc.err != kDevErrDepth) return fail(THV_EDEVICE, "batch device error %u", hc.err);
    return THV_OK;
  };

  // configuration: explicit, cached, autotuned on the first group, or default
  MsConfig cfg = kMsDefault;
  if (o && (o->small_degree || o->chunk_edges || o->mid_degree || o->small_group || o->mid_group)) {
    cfg.small = o->small_degree ? o->small_degree : kMsDefault.small;
    cfg.chunk = o->chunk_edges ? std::max<uint32_t>(32, (o->chunk_edges + 31) / 32 * 32) : kMsDefault.chunk;
    cfg.mid = o->mid_degree ? o->mid_degree : cfg.small;
    cfg.gsmall = o->small_group ? std::min<uint32_t>(o->small_group, 32) : kMsDefault.gsmall;
    cfg.gmid = o->mid_group ? std::min<uint32_t>(o->mid_group, 32) : kMsDefault.gmid;
  } else {
    const std::string key = tune_key(g, sssp);
    if (!tune_lookup(key, &cfg) && o && o->tune && n > 0) {
      // Coordinate descent over the buckets, one real group timed per
      // candidate: the chunk of the high-degree bucket, the small bucket's
      // boundary, the medium bucket (its upper boundary and vertices per
      // warp), the small bucket's vertices per warp, then threads per CTA.
      const uint32_t k = std::min(group, n);
      float best_ms = 1e30f;
      bool moot = false;
      auto trial = [&](MsConfig c) -> thv_status {
        if (moot) return THV_OK;
        if (c.mid < c.small) c.mid = c.small;
        float ms_ = 0;
        bool deep = false;
        THV_TRY(one_group(0, k, c, &ms_, &deep));
        if (deep) moot = true;  // depth fallback: tuning this graph is moot
        // a change has to win by 0.5%, above the run-to-run spread of one
        // group under one configuration (about 0.1%)
        else if (ms_ < best_ms * (best_ms < 1e29f ? 0.995f : 1.f)) { best_ms = ms_; cfg = c; }
        return THV_OK;
      };
      {
        // warm-up: the first pass pays for cold caches and first launches
        float ms_ = 0;
        bool deep = false;
        THV_TRY(one_group(0, k, kMsDefault, &ms_, &deep));
        moot = deep;
      }
      THV_TRY(trial(kMsDefault));
      // the two-bucket grid: small-bucket boundary x chunk size
      for (uint32_t sm : {16u, 64u, 256u})
        for (uint32_t ch : {256u, 512u, 1024u}) {
          MsConfig c = kMsDefault;
          c.small = c.mid = sm;
          c.chunk = ch;
          if (sm != kMsDefault.small || ch != kMsDefault.chunk) THV_TRY(trial(c));
        }
      {
        // a medium bucket above the small one, fewer vertices per warp
        const MsConfig base = cfg;
        for (uint32_t f : {4u, 16u}) {
          MsConfig c = base;
          c.mid = std::min(base.small * f, kMsMaxGroupedDeg);
          c.gmid = 4;
          if (c.mid > base.small) THV_TRY(trial(c));
        }
      }
      // lanes per vertex: the medium bucket always gets more than the small
      // one (fewer vertices per warp), 4 to 32
      if (cfg.mid > cfg.small) {
        const MsConfig base = cfg;
        for (uint32_t gm : {1u, 2u, 8u})
          if (gm < base.gsmall) { MsConfig c = base; c.gmid = gm; THV_TRY(trial(c)); }
      }
      {
        const MsConfig base = cfg;
        for (uint32_t gs : {16u, 8u})
          if (base.mid == base.small || gs > base.gmid) { MsConfig c = base; c.gsmall = gs; THV_TRY(trial(c)); }
      }
      { MsConfig c = cfg; c.threads = 256; THV_TRY(trial(c)); }
      tune_store(key, cfg);
    }
  }

  for (uint32_t first = 0; first < n; first += group) {
    const uint32_t k = std::min(group, n - first);
    float ms_ = 0.f;
    bool deep = false;
    THV_TRY(one_group(first, k, cfg, &ms_, &deep));
    if (deep) {
      // deeper than the u8 level bytes hold: this group one source at a time
      THV_TRY(fallback_single(g, sources + first, k, st, o, rows ? rows + first : nullptr,
                              checksums ? checksums + first : nullptr, local));
      continue;
    }
    dev_ms += ms_;
    const MsCtrl &hc = *b->h_ctrl;
    if (checksums) memcpy(checksums + first, b->h_sums, k * 8);
    local.iterations += hc.iters;
    local.edges_expanded += hc.edges;
    local.hbm_edge_bytes += hc.hbm_bytes;
    local.link_edge_bytes += hc.link_bytes;
    local.h2d_bytes += (kMsWidth + 1) * 4;
    uint64_t rows_out = 0;
    for (uint32_t i = 0; want_out && i < k; i++) rows_out += rows[first + i] != nullptr;
    local.d2h_bytes += sizeof(MsCtrl) + kMsWidth * 8 + rows_out * g->nv * 4;
  }
  local.device_ms += dev_ms;
  local.kernel_launches = launches;
  local.wall_ms = now_ms() - t0;
  if (stats) *stats = local;
  return THV_OK;
}

// ------------------------------------------------------ live groups (host)

// A joining BFS source needs this many levels of headroom below the u8
// level range; an SSSP source needs its shifted values below 2^32.
constexpr uint32_t kLiveBfsLevelRoom = 64;
constexpr uint64_t kLiveSsspRoom = 1ull << 24;

template <int OP, int ESZ, int THREADS>
static thv_status live_launch(thv_graph *g, MsArgs &a, cudaStream_t st) {
  BatchState *b = g->bs;
  auto kern = two_buckets(a) ? ms_kernel<OP, ESZ, THREADS, 32> : ms_kernel<OP, ESZ, THREADS, 0>;
  const size_t ring = OP == MS_SSSP ? (size_t)THREADS / 32 * kMsRing * 512 : 0;
  const size_t smem = ring + (g->plan.vbegin.size() <= kSmemBlocks + 1 ? g->plan.vbegin.size() * 4 : 0);
  THV_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int bpsm = 0;
  THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, THREADS, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "batch kernel cannot be resident");
  unsigned long long *alive = reinterpret_cast<unsigned long long *>(
      reinterpret_cast<char *>(b->d_ctrl) + offsetof(MsCtrl, alive));
  THV_CUDA(cudaMemsetAsync(alive, 0, 8, st));
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel((void *)kern, dim3(bpsm * g->num_sms), dim3(THREADS), args, smem, st));
  ms_alive<<<g->num_sms * 4, 256, 0, st>>>(a.front, a.nv, alive);
  THV_CUDA(cudaGetLastError());
  THV_CUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, sizeof(MsCtrl), cudaMemcpyDeviceToHost, st));
  return THV_OK;
}

template <int OP>
static thv_status live_launch_any(thv_graph *g, MsArgs &a, cudaStream_t st, uint32_t threads) {
  if (g->esz == 8)
    return threads == 256 ? live_launch<OP, 8, 256>(g, a, st) : live_launch<OP, 8, 512>(g, a, st);
  return threads == 256 ? live_launch<OP, 4, 256>(g, a, st) : live_launch<OP, 4, 512>(g, a, st);
}

static MsArgs live_args(thv_graph *g, const LiveGroup *lg, uint32_t timeout_ms) {
  MsArgs a = ms_args(g, g->bs, timeout_ms);
  a.delta = kMsDelta;
  a.growth = kMsGrowth;
  apply_config(a, MsConfig{lg->small, lg->chunk, lg->threads, lg->mid, lg->gsmall, lg->gmid});
  return a;
}

static thv_status live_state(thv_graph *g, const LiveGroup *lg) {
  if (!lg->bs || !lg->bs->valid) return fail(THV_EINVAL, "live group has no batch state");
  g->bs = lg->bs;
  return THV_OK;
}

thv_status live_open(thv_graph *g, LiveGroup *lg, bool sssp) {
  lg->sssp = sssp;
  lg->running = false;
  lg->active = 0;
  THV_TRY(dev_alloc((void **)&lg->d_buf, 4 * kMsWidth * 4, "live group staging"));
  THV_TRY(pinned_alloc((void **)&lg->h_buf, 4 * kMsWidth * 4, "live group staging"));
  THV_TRY(dev_alloc((void **)&lg->d_sums, kMsWidth * 8, "live group checksums"));
  THV_TRY(pinned_alloc((void **)&lg->h_sums, kMsWidth * 8, "live group checksums"));
  // each live group owns its traversal state, so several can be on the
  // device at once (the graph's own batch states serve thv_batch_run)
  lg->bs = new BatchState();
  return fill_batch_state(g, lg->bs, sssp, false);
}

void live_close(LiveGroup *lg) {
  free_state(lg->bs);
  dev_free(lg->d_buf);
  pinned_free(lg->h_buf);
  dev_free(lg->d_sums);
  pinned_free(lg->h_sums);
  lg->d_buf = lg->h_buf = nullptr;
  lg->d_sums = lg->h_sums = nullptr;
  lg->running = false;
  lg->active = 0;
}

bool live_can_join(const thv_graph *g, const LiveGroup *lg) {
  if (!lg->running) return true;
  if (__builtin_popcountll(lg->active) >= (int)kMsWidth) return false;
  if (!lg->sssp) return lg->level + kLiveBfsLevelRoom <= kMaxBfsLevel;
  return (uint64_t)lg->thr + g->nv + kLiveSsspRoom < 0xFFFFFFFFull;
}

thv_status live_add(thv_graph *g, LiveGroup *lg, uint32_t k, const uint32_t *sources,
                    uint32_t *bits, uint32_t timeout_ms, cudaStream_t st) {
  if (k == 0) return THV_OK;
  if ((uint32_t)__builtin_popcountll(lg->active) + k > kMsWidth)
    return fail(THV_EINVAL, "live group: %u sources do not fit", k);
  const bool fresh = !lg->running;
  if (fresh) {
    MsConfig cfg = kMsDefault;
    tune_lookup(tune_key(g, lg->sssp), &cfg);  // a configuration tuned by thv_batch_run
    lg->small = cfg.small;
    lg->chunk = cfg.chunk;
    lg->threads = cfg.threads;
    lg->mid = cfg.mid;
    lg->gsmall = cfg.gsmall;
    lg->gmid = cfg.gmid;
    lg->iter = 0;
    lg->level = 1;
    lg->width = kMsDelta;
    lg->thr = (uint32_t)std::min<uint64_t>(1ull + kMsDelta, 0xFFFFFFFFull);
    lg->active = 0;
  }
  THV_TRY(live_state(g, lg));
  BatchState *b = g->bs;
  MsArgs a = live_args(g, lg, timeout_ms);
  // value of the joining sources' vertices: BFS the level expanded next,
  // SSSP the lower end of the current window
  const uint32_t start = lg->sssp ? (uint32_t)std::max<int64_t>(1, (int64_t)lg->thr - lg->width)
                                  : lg->level;
  uint32_t *hb = lg->h_buf;  // [bits | sources | seed values | unreached per bit]
  unsigned long long jm = 0;
  uint32_t t = 0;
  for (uint32_t s = 0; s < kMsWidth && t < k; s++) {
    if ((lg->active >> s) & 1ull) continue;
    hb[t] = s;
    hb[kMsWidth + t] = sources[t];
    hb[2 * kMsWidth + t] = start;
    bits[t] = s;
    jm |= 1ull << s;
    lg->base[s] = start;
    t++;
  }
  for (uint32_t s = 0; s < kMsWidth; s++)
    hb[3 * kMsWidth + s] = (uint32_t)(g->nv + ((jm >> s) & 1ull ? start : 1u));
  THV_CUDA(cudaMemcpyAsync(lg->d_buf, hb, 4 * kMsWidth * 4, cudaMemcpyHostToDevice, st));
  const int igrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  if (fresh) {
    if (lg->sssp) ms_init<MS_SSSP><<<igrid, 256, 0, st>>>(a, b->ngroups * 32u);
    else ms_init<MS_BFS><<<igrid, 256, 0, st>>>(a, b->ngroups * 32u);
  } else {
    if (lg->sssp) ms_live_reset<MS_SSSP><<<igrid, 256, 0, st>>>(a, jm, lg->d_buf + 3 * kMsWidth);
    else ms_live_reset<MS_BFS><<<igrid, 256, 0, st>>>(a, jm, lg->d_buf + 3 * kMsWidth);
  }
  if (lg->sssp)
    ms_live_seed<MS_SSSP><<<1, kMsWidth, 0, st>>>(a, k, lg->d_buf, lg->d_buf + kMsWidth, lg->d_buf + 2 * kMsWidth);
  else
    ms_live_seed<MS_BFS><<<1, kMsWidth, 0, st>>>(a, k, lg->d_buf, lg->d_buf + kMsWidth, lg->d_buf + 2 * kMsWidth);
  THV_CUDA(cudaGetLastError());
  THV_CUDA(cudaStreamSynchronize(st));
  lg->active |= jm;
  lg->running = true;
  return THV_OK;
}

thv_status live_step(thv_graph *g, LiveGroup *lg, uint32_t iters, uint32_t timeout_ms,
                     cudaStream_t st, unsigned long long *finished, bool *too_deep) {
  *finished = 0;
  *too_deep = false;
  if (!lg->running || !lg->active) return THV_OK;
  THV_TRY(live_state(g, lg));
  BatchState *b = g->bs;
  MsArgs a = live_args(g, lg, timeout_ms);
  a.resume = 1;
  a.r_iter = lg->iter;
  a.r_level = lg->level;
  a.r_thr = lg->thr;
  a.r_width = lg->width;
  a.yield_at = lg->iter + std::max(iters, 1u);
  a.max_iters = 0xFFFFFFF0u;
  THV_TRY(lg->sssp ? live_launch_any<MS_SSSP>(g, a, st, lg->threads)
                   : live_launch_any<MS_BFS>(g, a, st, lg->threads));
  THV_CUDA(cudaStreamSynchronize(st));
  const MsCtrl &hc = *b->h_ctrl;
  if (hc.err == kDevErrDepth) {
    *too_deep = true;
    return THV_OK;
  }
  if (hc.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "grid barrier wait exceeded %u ms", timeout_ms);
  if (hc.err == kDevErrIters) return fail(THV_ETIMEOUT, "iteration cap reached");
  if (hc.err) return fail(THV_EDEVICE, "batch device error %u", hc.err);
  lg->edges = hc.edges;
  lg->hbm_bytes = hc.hbm_bytes;
  lg->link_bytes = hc.link_bytes;
  if (hc.yielded) {
    lg->iter = hc.y_iter;
    lg->level = hc.y_level;
    lg->thr = hc.y_thr;
    lg->width = hc.y_width;
    *finished = lg->active & ~hc.alive;
  } else {
    lg->iter = hc.iters;
    *finished = lg->active;  // no pending pair left: every source is done
  }
  return THV_OK;
}

thv_status live_collect(thv_graph *g, LiveGroup *lg, unsigned long long fin, uint64_t *sums,
                        uint32_t *const *out, uint32_t *d_stage, cudaStream_t st) {
  fin &= lg->active;
  if (!fin) return THV_OK;
  THV_TRY(live_state(g, lg));
  MsArgs a = live_args(g, lg, 60000u);
  uint32_t *hb = lg->h_buf + 3 * kMsWidth;
  for (uint32_t s = 0; s < kMsWidth; s++) hb[s] = (fin >> s) & 1ull ? lg->base[s] : 1u;
  THV_CUDA(cudaMemcpyAsync(lg->d_buf + 3 * kMsWidth, hb, kMsWidth * 4, cudaMemcpyHostToDevice, st));
  THV_CUDA(cudaMemsetAsync(lg->d_sums, 0, kMsWidth * 8, st));
  if (lg->sssp)
    ms_live_sums<MS_SSSP><<<g->num_sms * 8, kExtractThreads, 0, st>>>(a, fin, lg->d_buf + 3 * kMsWidth, lg->d_sums);
  else
    ms_live_sums<MS_BFS><<<g->num_sms * 8, kExtractThreads, 0, st>>>(a, fin, lg->d_buf + 3 * kMsWidth, lg->d_sums);
  THV_CUDA(cudaGetLastError());
  THV_CUDA(cudaMemcpyAsync(lg->h_sums, lg->d_sums, kMsWidth * 8, cudaMemcpyDeviceToHost, st));
  const int grid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  for (uint32_t s = 0; s < kMsWidth; s++) {
    if (!((fin >> s) & 1ull) || !out || !out[s]) continue;
    if (lg->sssp) ms_live_column<MS_SSSP><<<grid, 256, 0, st>>>(a, s, lg->base[s], d_stage);
    else ms_live_column<MS_BFS><<<grid, 256, 0, st>>>(a, s, lg->base[s], d_stage);
    THV_CUDA(cudaGetLastError());
    THV_CUDA(cudaMemcpyAsync(out[s], d_stage, g->nv * 4, cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaStreamSynchronize(st));  // d_stage is reused by the next source
  }
  THV_CUDA(cudaStreamSynchronize(st));
  for (uint32_t s = 0; s < kMsWidth; s++)
    if ((fin >> s) & 1ull) sums[s] = lg->h_sums[s];
  lg->active &= ~fin;
  if (!lg->active) lg->running = false;
  return THV_OK;
}

}  // namespace thv
