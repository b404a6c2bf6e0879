// Frontier engine for the monotone min-propagation family: BFS, CC, SSSP.
//
// Replaces the reference's per-level host loop (src/bfs/bfs.cu:55-524,
// src/cc/cc.cu:71-614, src/sssp/sssp.cu:10-570) and its static / demand /
// filter kernels (src/bfs/bfs_kernels.cu:4-287, src/cc/cc_kernels.cu:4-269,
// src/sssp/sssp_kernels.cu:4-229) with ONE persistent cooperative kernel:
//
//   iteration i:
//     compaction  - scan the pending-vertex bitmap 32 words per warp; ballot /
//                   popc compaction of the taken vertices into two work
//                   queues: "small" vertices (degree < small_degree), served
//                   32 per warp with warp-cooperative load balancing, and
//                   fixed-size edge chunks of high-degree vertices, one chunk
//                   per warp with 128-byte aligned 16-byte vector loads.  A
//                   word with no pending vertex costs one load: whole edge
//                   blocks without an active source are never touched.
//     grid barrier
//     expansion   - warps pull tasks from an atomic counter; each edge does
//                   "if (cand < val[w]) atomicMin; mark w pending".
//     grid barrier
//
// The relaxation is the reference's (bfs_kernels.cu:63-70: new value < old
// => atomicMin + frontier flag).  Its fixed point is unique, so results are
// bit-exact whatever the schedule: BFS level+1, CC min reaching id, SSSP
// min(dist+1, n+1).  SSSP takes only pending vertices below a moving
// threshold (near/far split) to avoid re-expanding vertices whose distance
// is still falling -- each re-expansion of a non-resident vertex re-reads
// its adjacency over the host link.  A per-bitmap-word lower bound of the
// pending values lets the compaction skip words that hold only far
// vertices without reading their values.
//
// Each vertex's adjacency is addressed through its edge block's base
// address: resident blocks point into the HBM buffer, the others into the
// pinned, mapped host copy, which the same load instructions read over the
// host link (zero copy).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

enum { OP_BFS = 0, OP_CC = 1, OP_SSSP = 2 };

constexpr int kMinThreads = 512;
constexpr uint32_t kDefaultSmall = 64;  // degree < this: warp-cooperative
// Queue mode: HBM lists of degree < this go to the small-vertex groups
// (lists read over the link always go to chunk items).  RMAT-24 SSSP, 40%
// HBM, sources 1 / 7 / 1000 / 2: 64 5.58 / 6.91 / 7.35 / 6.44 ms, 128 5.46
// / 6.55 / 6.92 / 6.10, 256 5.40 / 6.50 / 6.84 / 6.04.
constexpr uint32_t kQueueSmall = 256;
constexpr uint32_t kDefaultChunk = 256; // edges per high-degree work item
// Queue mode: one warp in this many (the link warps) drains the host-list
// chunks of a phase first.  RMAT-24 SSSP, 40% HBM, mean over sources 1, 2,
// 7 and 1000: every 3rd warp 7.41 ms, 4th 6.75, 5th 6.60, 6th 6.61, 8th
// 6.90 (source 1: 6.23, 5.78, 5.68, 5.60, 5.56; every 16th: 6.24).  All
// chunks in queue order took 5.96 / 7.73 / 8.18 ms at sources 1 / 7 / 1000
// (every 6th: 5.60 / 6.95 / 7.43); no link warps (host chunks last) 7.27
// ms at source 1.
constexpr uint32_t kLinkEvery = 6;
constexpr uint32_t kQueueChunkBytes = 4096;  // queue mode: bytes of edges per item (4 steps of 8 edges per lane when packed)
// scan mode (BFS, CC): RMAT-20 BFS 0.408 -> 0.40 ms and RMAT-24 label
// propagation 31.2 -> 30.1 ms with 1024 4-byte edges per item instead of 256
constexpr uint32_t kScanChunkBytes = 4096;
// SSSP near/far width.  Measured at RMAT-24 (40% in HBM): width 2 expands
// every vertex once (link bytes = algorithmic) but needs ~200 iterations;
// width 8 re-reads 5% more adjacency in ~80 iterations and is fastest.
constexpr uint32_t kDefaultDelta = 8;
constexpr uint32_t kCcGrowth = 8;       // CC label window growth per advance
// SSSP window growth per advance.  RMAT-24 (40% HBM budget), window 8:
// fixed windows need 85 iterations and ~20 bitmap scans; growth 8 needs 19
// iterations for the same edges expanded (10.4 -> 7.7 ms); growth 16 (18
// iterations) measured 1.3% faster than 8 over ten sources.  With the link
// warps, at sources 1 / 7 / 1000 / 2: growth 8 5.61 / 7.02 / 7.40 / 6.60
// ms, 16 5.56 / 6.92 / 7.37 / 6.45, 32 5.52 / 6.88 / 7.33 / 6.42 (15
// iterations), 64 5.52 / 6.90 / 7.30 / 6.42.
constexpr uint32_t kSsspGrowth = 32;
// Direction-optimising BFS switch factors (Beamer et al., SC'12): go
// bottom-up when the frontier's out-edges exceed the unexplored edges /
// alpha, back to top-down when the frontier falls below nv / beta.  Alpha 4
// instead of the paper's 14: on RMAT-20..24 sources, 14 and 30 sometimes
// switch a level early and scan 4-8x more in-edges (0.38 vs 0.73 ms).
constexpr uint32_t kBfsAlpha = 4, kBfsBeta = 24;
// Bottom-up BFS: in-edges (and their frontier words) loaded at once per
// lane.
constexpr int kBuBatch = 4;
// Direction-optimising BFS: a top-down level whose frontier holds at most
// this many vertices and out-edges runs inside one CTA, with block
// barriers, and so do the levels after it while they stay that small.
constexpr uint32_t kLocalCap = 2048;


// Frontier work item of the single-source engine: the adjacency of vertex v
// (or one chunk of it) plus v's value when it was taken, so the expansion
// needs no dependent load of val[v] (a value that fell since is a larger,
// still valid bound, and the fall re-queued v).  Edge addresses fit in 48
// bits (checked on the host); the edge count takes the top 16.
struct __align__(16) MinItem {
  unsigned long long ea_cnt;
  uint32_t v, val;
};
constexpr unsigned long long kAddrMask = (1ull << 48) - 1;
__device__ __forceinline__ MinItem make_item(unsigned long long ea, uint32_t cnt, uint32_t v,
                                             uint32_t val) {
  return MinItem{ea | ((unsigned long long)cnt << 48), v, val};
}

struct MinCtrl {
  GridBar bar;
  unsigned err, iters;
  unsigned long long cnt_small[3], cnt_big[3], remaining[3], wc[3];
  unsigned minkept[3], pad;
  unsigned long long edges, hbm_bytes, link_bytes, vertices;
  unsigned long long checksum;
  // BFS: out-edges and size of each level's frontier; bottom-up levels run
  unsigned long long mf[3], nf[3], bu_scan[3];
  unsigned bu_levels, pad2;
  // queue mode: chunk items of host-resident lists (counted apart, stored
  // from the top of the chunk queue down) and their work counters
  unsigned long long cnt_host[3], wc_host[3];
  // direction-optimising BFS: vertices found per level while the level is
  // small enough to list them, and what a run of one-CTA levels hands back
  unsigned fl_cnt[3], loc_levels;
  unsigned long long loc_mu;
};

struct MinArgs {
  uint32_t *val;
  uint32_t *bm;
  uint32_t *wmin;  // SSSP/CC: lower bound of the pending values in each bitmap word;
                   // BFS (may be null): per-group counters of the compaction
  const uint64_t *off;
  const uint32_t *blk_vb;
  const uint64_t *blk_base;
  uint64_t host_base, host_end;  // zero-copy edge range [host_base, host_end)
  ListCache lc;
  unsigned long long *blk_access;  // tracked plans: adjacency bytes read per block
  MinItem *qs, *qb;
  unsigned long long cap_s, cap_b;
  MinCtrl *ctrl;
  // queue mode: second queue buffers and two queued-vertex bitmaps (one
  // per phase parity, ngroups * 32 words each)
  MinItem *qs2, *qb2;
  uint32_t *qbits;
  unsigned long long timeout_ns;
  uint32_t nblk, nv, ngroups, max_iters;
  uint32_t delta, small_deg, chunk, src;
  uint32_t growth;
  uint32_t wshift, wbase;  // packed weighted edges (see edge_dst / edge_wt)
  uint32_t pad;
  // direction-optimising BFS: in-edge transpose, frontier copy, switch
  // factors (do_alpha = 0: top-down only)
  const uint64_t *in_off;
  const uint32_t *in_adj;
  uint32_t *bm2;
  unsigned long long ne;
  uint32_t do_alpha, do_beta;
  // queue mode: one warp in link_every draws host-list chunks first (0: none)
  uint32_t link_every, pad3;
  // direction-optimising BFS: lists of small frontiers (3 slots of
  // kLocalCap vertices)
  uint32_t *flist;
};

struct MinState {
  uint64_t nv = 0;
  uint32_t *d_val = nullptr;
  uint32_t *d_bm = nullptr;
  uint32_t *d_wmin = nullptr;
  uint32_t *d_bm2 = nullptr;  // BFS frontier copy for bottom-up levels
  uint32_t *d_flist = nullptr;  // BFS small-frontier lists
  MinItem *d_qs = nullptr, *d_qb = nullptr;
  MinItem *d_qs2 = nullptr, *d_qb2 = nullptr;
  uint32_t *d_qbits = nullptr;
  uint64_t cap_s = 0, cap_b = 0;
  uint32_t chunk = 0, small = 0;
  MinCtrl *d_ctrl = nullptr;
  MinCtrl *h_ctrl = nullptr;  // pinned
  uint32_t ngroups = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool valid = false;
};

// Position of the n-th (from 0) set bit of x; n < popc(x).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t n) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t s = 16; s > 0; s >>= 1) {
    const uint32_t lo = __popc(x & ((1u << s) - 1u));
    if (n >= lo) {
      n -= lo;
      x >>= s;
      pos += s;
    }
  }
  return pos;
}

template <int OP>
__device__ __forceinline__ void activate(const MinArgs &a, uint32_t w,
                                         unsigned long long cand) {
  if (OP != OP_BFS) atomicMin(a.wmin + (w >> 5), (uint32_t)cand);
  const uint32_t m = 1u << (w & 31u);
  uint32_t *bp = a.bm + (w >> 5);
  if (!(ldcg(bp) & m)) atomicOr(bp, m);
}

// Direction-optimising BFS keeps the frontier double-buffered: a vertex
// found at this level goes into `bits` (the next level's bitmap), and the
// next level's size and out-edges are counted as vertices are found, so the
// next level's direction is known before any of its work.
struct NextLevel {
  uint32_t *bits;
  unsigned long long nf, mf;
  uint32_t *list;      // found vertices are listed here too (or null)
  unsigned *list_cnt;  // their count; the level's out-edges bound it by kLocalCap
};

// Relax N edges at once: all value probes are issued before any atomic so a
// lane keeps N loads in flight.  NEXT (BFS): mark found vertices in nl->bits
// and count them and their out-edges.
template <int OP, int N, bool NEXT = false>
__device__ __forceinline__ void relax_n(const MinArgs &a, const uint32_t (&w)[N],
                                        const unsigned long long (&cand)[N],
                                        const bool (&ok)[N], NextLevel *nl = nullptr) {
  uint32_t cur[N];
#pragma unroll
  for (int j = 0; j < N; j++) cur[j] = ok[j] ? ldcg(a.val + w[j]) : 0u;
  if constexpr (NEXT) {
    bool found[N];
#pragma unroll
    for (int j = 0; j < N; j++)
      found[j] = ok[j] && cand[j] < cur[j] && cand[j] < atomicMin(a.val + w[j], (uint32_t)cand[j]);
    uint32_t deg[N];
#pragma unroll
    for (int j = 0; j < N; j++)
      deg[j] = found[j] ? (uint32_t)(__ldg(a.off + w[j] + 1) - __ldg(a.off + w[j])) : 0u;
#pragma unroll
    for (int j = 0; j < N; j++) {
      if (!found[j]) continue;
      const uint32_t m = 1u << (w[j] & 31u);
      uint32_t *bp = nl->bits + (w[j] >> 5);
      if (!(ldcg(bp) & m)) atomicOr(bp, m);
      nl->nf++;
      nl->mf += deg[j];
      if (nl->list) nl->list[atomicAdd(nl->list_cnt, 1u)] = w[j];
    }
  } else {
#pragma unroll
    for (int j = 0; j < N; j++) {
      if (ok[j] && cand[j] < cur[j]) {
        const uint32_t old = atomicMin(a.val + w[j], (uint32_t)cand[j]);
        if (cand[j] < old) activate<OP>(a, w[j], cand[j]);
      }
    }
  }
}

__device__ __forceinline__ uint32_t sat32(unsigned long long x) {
  return x > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)x;
}

template <int OP>
__device__ __forceinline__ unsigned long long candidate(uint32_t vval, uint32_t wt) {
  return OP == OP_BFS    ? (unsigned long long)vval + 1ull
         : OP == OP_SSSP ? (unsigned long long)vval + wt
                         : (unsigned long long)vval;
}

// One high-degree chunk (or part `part` of `parts` of it) per warp:
// 128-byte aligned 16-byte loads, two per lane in flight, lanes outside
// [start, end) masked.
template <int OP, int ESZ, bool NEXT = false>
__device__ __forceinline__ void process_chunk(const MinArgs &a, const MinItem &it, unsigned part,
                                              unsigned parts, NextLevel *nl = nullptr) {
  constexpr int PER = 16 / ESZ;  // edges per 16-byte load
  const unsigned lane = lane_id();
  const uint32_t vval = it.val;
  const uint32_t cnt = (uint32_t)(it.ea_cnt >> 48);
  // parts of whole 32-edge runs
  const uint32_t per = ((cnt + parts - 1) / parts + 31u) & ~31u;
  const uint32_t lo = min(cnt, part * per), hi = min(cnt, lo + per);
  const uintptr_t start = (it.ea_cnt & kAddrMask) + (uintptr_t)lo * ESZ;
  const uintptr_t end = (it.ea_cnt & kAddrMask) + (uintptr_t)hi * ESZ;
  for (uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane; p < end; p += 1024u) {
    uint4 q[2];
    q[0] = ld_nc_v4(p);
    const bool second = p + 512u < end;
    q[1] = second ? ld_nc_v4(p + 512u) : make_uint4(0, 0, 0, 0);
    uint32_t w[2 * PER];
    unsigned long long cand[2 * PER];
    bool ok[2 * PER];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uintptr_t ph = p + 512u * h;
      const uint32_t f[4] = {q[h].x, q[h].y, q[h].z, q[h].w};
#pragma unroll
      for (int j = 0; j < PER; j++) {
        const uintptr_t ea = ph + (uintptr_t)ESZ * j;
        const int k = h * PER + j;
        ok[k] = (h == 0 || second) && ea >= start && ea < end;
        w[k] = ESZ == 4 ? edge_dst(f[j], a.wshift) : f[2 * j];
        cand[k] = candidate<OP>(vval, ESZ == 4 ? edge_wt(f[j], a.wshift, a.wbase) : f[2 * j + 1]);
      }
    }
    relax_n<OP, 2 * PER, NEXT>(a, w, cand, ok, nl);
  }
}

// Scan-mode small-vertex groups: edges per lane in flight per step.
constexpr int kScanGroupPer = 4;

// Up to 32 (gsize) low-degree vertices per warp: warp-cooperative load
// balancing over their concatenated adjacency, kScanGroupPer x 32 edges per
// step (each lane's edges in flight together).
template <int OP, int ESZ, bool NEXT = false>
__device__ __forceinline__ void process_group(const MinArgs &a, unsigned long long first,
                              unsigned long long n_small, unsigned gsize = 32,
                              NextLevel *nl = nullptr) {
  constexpr int P = kScanGroupPer;
  const unsigned lane = lane_id();
  const unsigned long long idx = first + lane;
  MinItem it{0, 0, 0};
  if (lane < gsize && idx < n_small) it = a.qs[idx];
  const uint32_t vval = it.val;
  const unsigned cnt = (unsigned)(it.ea_cnt >> 48);
  const unsigned long long eaddr = it.ea_cnt & kAddrMask;
  const unsigned incl = warp_incl_scan<unsigned>(cnt);
  const unsigned excl = incl - cnt;
  const unsigned total = __shfl_sync(kFull, incl, 31);
  for (unsigned k = 0; k < total; k += 32u * P) {
    uint32_t w[P];
    unsigned long long cand[P];
    bool ok[P];
    uintptr_t addr[P];
    uint32_t ov[P];
#pragma unroll
    for (int h = 0; h < P; h++) {
      const unsigned t = k + 32u * h + lane;
      const int o = warp_owner(excl, t);
      const unsigned long long ea = shfl64(eaddr, o);
      const unsigned oex = __shfl_sync(kFull, excl, o);
      ov[h] = __shfl_sync(kFull, vval, o);
      ok[h] = t < total;
      addr[h] = (uintptr_t)ea + (uintptr_t)(t - oex) * ESZ;
    }
    uint32_t wt[P];
#pragma unroll
    for (int h = 0; h < P; h++) {
      if (ESZ == 4) {
        const uint32_t e = ok[h] ? ld_nc_u32(addr[h]) : 0u;
        w[h] = edge_dst(e, a.wshift);
        wt[h] = edge_wt(e, a.wshift, a.wbase);
      } else {
        const uint2 e = ok[h] ? ld_nc_u2(addr[h]) : make_uint2(0, 0);
        w[h] = e.x;
        wt[h] = e.y;
      }
    }
#pragma unroll
    for (int h = 0; h < P; h++) cand[h] = candidate<OP>(ov[h], wt[h]);
    relax_n<OP, P, NEXT>(a, w, cand, ok, nl);
  }
}

// Bottom-up BFS level: every unreached vertex scans its in-edges for a
// parent in this level's frontier `front`, stopping at the first.  A warp
// owns 32 vertices (one bitmap word) at a time, so the next frontier word is
// its ballot, stored whole into `next`.  value = level + 1 for the vertices
// reached here; their number and out-edges go to *next_nf / *next_mf.
// (Scalar arguments: a MinArgs reference would copy the kernel's
// parameter block to local memory.)
__device__ __noinline__ void bfs_bottom_up(const uint64_t *in_off, const uint32_t *in_adj,
                                           const uint64_t *off, const uint32_t *front,
                                           uint32_t *next, uint32_t *val, uint32_t nv,
                                           uint32_t value, unsigned long long *edges,
                                           unsigned long long *level_scan,
                                           unsigned long long *next_nf,
                                           unsigned long long *next_mf, unsigned gwarp,
                                           unsigned nwarps) {
  const unsigned lane = lane_id();
  const uint32_t nwords = (nv + 31) / 32;
  unsigned long long scanned = 0, nf = 0, mf = 0;
  // a vertex's value, in-edge range and out-edge range load together, and
  // those of the warp's next word load before this word's scan
  uint32_t nval = 0;
  uint64_t ns = 0, ne = 0, nos = 0, noe = 0;
  auto prefetch = [&](uint32_t w) {
    const uint32_t v = w * 32u + lane;
    if (w < nwords && v < nv) {
      nval = ldcg(val + v);
      ns = __ldg(in_off + v);
      ne = __ldg(in_off + v + 1);
      nos = __ldg(off + v);
      noe = __ldg(off + v + 1);
    } else {
      nval = 0;  // not a vertex: nothing to scan
    }
  };
  prefetch(gwarp);
  for (uint32_t w = gwarp; w < nwords; w += nwarps) {
    const uint32_t v = w * 32u + lane;
    const uint32_t cval = nval;
    const uint64_t s = ns, e = ne, os = nos, oe = noe;
    prefetch(w + nwarps);
    bool found = false;
    if (v < nv && cval == nv + 1u) {
      // kBuBatch in-edges and then their frontier words in flight at once
      // (one load pair per edge in turn made a lane's scan a chain of
      // dependent round trips); edges count up to the parent found
      for (uint64_t k = s; k < e && !found; k += kBuBatch) {
        uint32_t u[kBuBatch], fw[kBuBatch];
#pragma unroll
        for (int j = 0; j < kBuBatch; j++) u[j] = k + j < e ? __ldg(in_adj + k + j) : 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < kBuBatch; j++)
          fw[j] = u[j] != 0xFFFFFFFFu ? ldcg(front + (u[j] >> 5)) : 0u;
#pragma unroll
        for (int j = 0; j < kBuBatch; j++) {
          if (!found && u[j] != 0xFFFFFFFFu) {
            scanned++;
            found = (fw[j] >> (u[j] & 31u)) & 1u;
          }
        }
      }
      if (found) {
        val[v] = value;
        nf++;
        mf += oe - os;
      }
    }
    const unsigned fm = __ballot_sync(kFull, found);
    if (lane == 0) next[w] = fm;
  }
  scanned = warp_sum(scanned);
  nf = warp_sum(nf);
  mf = warp_sum(mf);
  if (lane == 0) {
    if (scanned) {
      atomicAdd(edges, scanned);
      atomicAdd(level_scan, scanned);
    }
    if (nf) {
      atomicAdd(next_nf, nf);
      atomicAdd(next_mf, mf);
    }
  }
}

// Top-down BFS levels inside one CTA (its threads only; the other CTAs
// wait at the grid barrier).  The frontier of the first level is the list
// `list_in` (n_in <= kLocalCap vertices, value lv); its bits are cleared
// from F, each level relaxes its out-edges (at most kLocalCap) edge-parallel
// over the block, found vertices (value lv + 1, ...) form the next list in
// shared memory, and the run stops at a frontier that is empty, holds more
// than kLocalCap out-edges, or would go bottom-up (out-edges x alpha above
// the unexplored edges).  That frontier's bits are set in F and its size and
// out-edges returned; *levels counts the levels run, *edges their
// out-edges, and *mu comes back with the out-edges of every frontier after
// the first and before the last taken off (as the grid's levels do).
// Scalar arguments: a MinArgs reference would copy the kernel's parameter
// block to local memory.
template <int ESZ>
__device__ __noinline__ void bfs_local_levels(const uint64_t *off, const uint32_t *vb,
                                              const unsigned long long *bbase, uint32_t nblk,
                                              uint32_t wshift, uint32_t *val, uint32_t *F,
                                              const uint32_t *list_in, uint32_t n_in,
                                              uint32_t src, uint32_t lv, uint32_t alpha,
                                              unsigned long long *mu, unsigned *levels,
                                              unsigned long long *edges, unsigned *nf_out,
                                              unsigned long long *mf_out) {
  __shared__ uint32_t s_fr[2][kLocalCap];
  __shared__ unsigned long long s_ea[kLocalCap];
  __shared__ uint32_t s_pre[kLocalCap + 1];
  __shared__ uint32_t s_wsum[32];
  __shared__ uint32_t s_n;
  __shared__ unsigned long long s_mf;
  const unsigned tid = threadIdx.x, nt = blockDim.x, lane = lane_id(), warp = tid >> 5;
  for (uint32_t i = tid; i < n_in; i += nt) {
    const uint32_t v = list_in ? list_in[i] : src;  // no list: the source alone
    s_fr[0][i] = v;
    atomicAnd(F + (v >> 5), ~(1u << (v & 31u)));
  }
  unsigned cur = 0, run = 0;
  uint32_t n = n_in;
  unsigned long long m = *mu, ed = 0, mf_next = 0;
  for (;;) {
    if (tid == 0) {
      s_n = 0;
      s_mf = 0;
    }
    __syncthreads();
    // degrees and list addresses of this frontier; exclusive scan of the
    // degrees, kLocalCap / blockDim.x consecutive entries per thread
    const uint32_t per = (kLocalCap + nt - 1) / nt;
    const uint32_t i0 = tid * per;
    uint32_t dsum = 0;
    for (uint32_t i = i0; i < i0 + per && i < n; i++) {
      const uint32_t v = s_fr[cur][i];
      const uint64_t s0 = __ldg(off + v), e0 = __ldg(off + v + 1);
      s_pre[i] = (uint32_t)(e0 - s0);
      s_ea[i] = bbase[find_block(vb, nblk, v)] + s0 * ESZ;
      dsum += (uint32_t)(e0 - s0);
    }
    const uint32_t incl = warp_incl_scan<uint32_t>(dsum);
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t x = lane < nt / 32 ? s_wsum[lane] : 0u;
      const uint32_t xi = warp_incl_scan<uint32_t>(x);
      if (lane < nt / 32) s_wsum[lane] = xi - x;
    }
    __syncthreads();
    uint32_t run_sum = s_wsum[warp] + incl - dsum;
    for (uint32_t i = i0; i < i0 + per && i < n; i++) {
      const uint32_t d = s_pre[i];
      s_pre[i] = run_sum;
      run_sum += d;
    }
    if (tid == nt - 1) s_pre[n] = run_sum;  // the last thread's end is the total
    __syncthreads();
    const uint32_t total = s_pre[n];
    // edge-parallel relaxation: edge e belongs to the last vertex o with
    // s_pre[o] <= e
    for (uint32_t e = tid; e < total; e += nt) {
      uint32_t lo = 0, hi = n;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_pre[mid] <= e) lo = mid;
        else hi = mid;
      }
      const uintptr_t ea = (uintptr_t)s_ea[lo] + (uintptr_t)(e - s_pre[lo]) * ESZ;
      const uint32_t raw = ld_nc_u32(ea);
      const uint32_t w = ESZ == 4 ? edge_dst(raw, wshift) : raw;
      if (ldcg(val + w) > lv + 1u && atomicMin(val + w, lv + 1u) > lv + 1u)
        s_fr[cur ^ 1u][atomicAdd(&s_n, 1u)] = w;  // at most total <= kLocalCap
    }
    __syncthreads();
    const uint32_t nn = s_n;
    unsigned long long mfl = 0;
    for (uint32_t i = tid; i < nn; i += nt) {
      const uint32_t w = s_fr[cur ^ 1u][i];
      mfl += __ldg(off + w + 1) - __ldg(off + w);
    }
    mfl = warp_sum(mfl);
    if (lane == 0 && mfl) atomicAdd(&s_mf, mfl);
    __syncthreads();
    mf_next = s_mf;
    ed += total;
    run++;
    const unsigned long long m_next = m > mf_next ? m - mf_next : 0ull;
    if (nn == 0 || mf_next > kLocalCap || mf_next * alpha > m_next) {
      // hand the frontier back to the grid as bits
      for (uint32_t i = tid; i < nn; i += nt) {
        const uint32_t w = s_fr[cur ^ 1u][i];
        atomicOr(F + (w >> 5), 1u << (w & 31u));
      }
      *nf_out = nn;
      break;
    }
    m = m_next;
    n = nn;
    cur ^= 1u;
    lv++;
    __syncthreads();
  }
  *mu = m;
  *levels = run;
  *edges = ed;
  *mf_out = mf_next;
}

// Direction-optimising BFS on a graph whose out-edges are all resident,
// with an in-edge transpose in HBM.  The frontier is double-buffered (F:
// this level's, N: the next one's), and each level's direction is decided
// before any of its work, from its frontier's size and out-edges, which the
// previous level counted while it found those vertices (Beamer et al.,
// SC'12: bottom-up when the frontier's out-edges exceed the unexplored
// edges / alpha; top-down again when the frontier holds fewer than nv / beta
// vertices, or its out-edges fall below half of what the last bottom-up
// level scanned).  A top-down level compacts F into work queues (clearing N
// on the way) and expands them, marking found vertices in N: two grid
// barriers.  A bottom-up level is one sweep that writes N whole: one
// barrier, and no compaction at all.  Levels are unique, so the values are
// bit-exact whatever the direction.
template <int ESZ>
__global__ void __launch_bounds__(kMinThreads, 2) bfs_do_kernel(MinArgs a) {
  extern __shared__ unsigned long long s_tab[];
  const bool smem_tab = a.nblk <= kSmemBlocks;
  unsigned long long *s_base = s_tab;
  uint32_t *s_vb = reinterpret_cast<uint32_t *>(s_tab + a.nblk);
  if (smem_tab) {
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];
    for (uint32_t i = threadIdx.x; i < a.nblk; i += blockDim.x) s_base[i] = a.blk_base[i];
  }
  __syncthreads();
  const uint32_t *vb = smem_tab ? s_vb : a.blk_vb;
  const unsigned long long *bbase = smem_tab ? s_base : (const unsigned long long *)a.blk_base;
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  // fewer bitmap groups than warps: nsub warps share a group, each taking
  // every nsub-th step of its numbered vertices (F is only read here)
  const unsigned nsub = a.ngroups * 2u <= nwarps ? min(8u, nwarps / a.ngroups) : 1u;
  const unsigned gstride = nwarps / nsub, sub = gwarp % nsub;
  uint32_t *F = a.bm, *N = a.bm2;
  unsigned long long mu = a.ne;      // out-edges of vertices not yet reached
  unsigned long long last_scan = 0;  // in-edges scanned by the last bottom-up level
  bool bottom_up = false;
  bool listed = false;  // the last level listed the vertices it found
  const unsigned long long src_deg = __ldg(a.off + a.src + 1) - __ldg(a.off + a.src);
  unsigned iter = 0;
  for (;; ++iter) {
    if (iter >= a.max_iters) {
      if (leader) atomicCAS(&c->err, 0u, kDevErrIters);
      break;
    }
    // Counter slots.  Level L compacts into slot L % 3 and counts level
    // L+1's frontier into (L + 1) % 3, which is read at the top of level
    // L + 1.  Slot (L + 2) % 3 of those counters was last read before level
    // L - 1's last barrier and is next written during level L + 1, so it is
    // cleared now.  The bottom-up scan count of level L (slot L % 3) is read
    // just after level L's last barrier, so it is cleared one level ahead
    // instead: slot (L + 1) % 3, last read after level L - 2's barrier.
    const unsigned slot = iter % 3, nslot = (iter + 1) % 3, zslot = (iter + 2) % 3;
    if (leader) {
      c->cnt_small[zslot] = 0;
      c->cnt_big[zslot] = 0;
      c->wc[zslot] = 0;
      c->mf[zslot] = 0;
      c->nf[zslot] = 0;
      c->fl_cnt[zslot] = 0;
      c->bu_scan[nslot] = 0;
    }
    const unsigned long long nf = iter == 0 ? 1ull : ldcg(&c->nf[slot]);
    const unsigned long long mf = iter == 0 ? src_deg : ldcg(&c->mf[slot]);
    if (nf == 0) break;
    mu = mu > mf ? mu - mf : 0;
    bottom_up = bottom_up ? nf * a.do_beta >= a.nv && 2 * mf > last_scan : mf * a.do_alpha > mu;
    const uint32_t lval = iter + 1u;  // value of this level's vertices
    if (!bottom_up && a.flist && (iter == 0 || listed) && nf <= kLocalCap && mf <= kLocalCap) {
      // a small top-down level (and the small ones after it) in CTA 0,
      // while the others wait at one grid barrier instead of two per level
      if (blockIdx.x == 0) {
        unsigned long long lmu = mu, led = 0, lmf = 0;
        unsigned lk = 0, lnf = 0;
        bfs_local_levels<ESZ>(a.off, vb, bbase, a.nblk, a.wshift, a.val, F,
                              iter == 0 ? nullptr : a.flist + slot * kLocalCap, (uint32_t)nf,
                              a.src, lval, a.do_alpha, &lmu, &lk, &led, &lnf, &lmf);
        if (threadIdx.x == 0) {
          atomicAdd(&c->edges, led);
          atomicAdd(&c->hbm_bytes, led * ESZ);  // every list is resident here
          // the grid resumes at level iter + lk with clean counters and
          // that level's frontier size and out-edges in its slot
          for (int k = 0; k < 3; k++) {
            c->cnt_small[k] = 0;
            c->cnt_big[k] = 0;
            c->wc[k] = 0;
            c->mf[k] = 0;
            c->nf[k] = 0;
            c->bu_scan[k] = 0;
            c->fl_cnt[k] = 0;
          }
          c->nf[(iter + lk) % 3] = lnf;
          c->mf[(iter + lk) % 3] = lmf;
          c->loc_levels = lk;
          c->loc_mu = lmu;
        }
      }
      if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
      mu = ldcg(&c->loc_mu);
      iter += ldcg(&c->loc_levels) - 1u;  // the loop's ++iter completes the jump
      listed = false;
      continue;  // F already holds the next level's frontier
    }
    if (bottom_up) {
      bfs_bottom_up(a.in_off, a.in_adj, a.off, F, N, a.val, a.nv, lval + 1u, &c->edges,
                    &c->bu_scan[slot], &c->nf[nslot], &c->mf[nslot], gwarp, nwarps);
      if (leader) c->bu_levels++;
      if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
      last_scan = ldcg(&c->bu_scan[slot]);
      listed = false;
    } else {
      if (leader) atomicAdd(&c->edges, mf);
      // ------------------------------------------------------ compaction
      unsigned long long my_hbm = 0, my_link = 0;
      for (unsigned g = gwarp / nsub; g < a.ngroups && gwarp / nsub < gstride; g += gstride) {
        const unsigned wbase = g * 32u;
        const uint32_t word = ldcg(F + wbase + lane);
        if (sub == 0) N[wbase + lane] = 0;
        const unsigned cnt = (unsigned)__popc(word);
        const unsigned incl = warp_incl_scan<unsigned>(cnt);
        const unsigned excl = incl - cnt, total = __shfl_sync(kFull, incl, 31);
        for (unsigned k = 32u * sub; k < total; k += 32u * nsub) {
          const unsigned t = k + lane;
          const int own = warp_owner(excl, t);
          const uint32_t ow = __shfl_sync(kFull, word, own);
          const unsigned oex = __shfl_sync(kFull, excl, own);
          const bool take = t < total;
          const uint32_t v = take ? (wbase + own) * 32u + nth_set_bit(ow, t - oex) : 0u;
          uint32_t deg = 0;
          unsigned long long eaddr = 0;
          if (take) {
            const uint64_t s0 = __ldg(a.off + v), e0 = __ldg(a.off + v + 1);
            deg = (uint32_t)(e0 - s0);
            bool host;
            const uint32_t bi = find_block(vb, a.nblk, v);
            eaddr = list_addr(a.lc, bbase[bi], a.host_base, v, s0, deg, ESZ, &host);
            if (a.blk_access) atomicAdd(a.blk_access + bi, (unsigned long long)deg * ESZ);
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
              if (pos < a.cap_s) a.qs[pos] = make_item(eaddr, deg, v, lval);
              else atomicCAS(&c->err, 0u, kDevErrQueue);
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
              for (unsigned kk = 0; kk < nch; kk++, pos++) {
                const uint32_t lo = kk * a.chunk;
                if (pos < a.cap_b)
                  a.qb[pos] = make_item(eaddr + (unsigned long long)lo * ESZ, min(a.chunk, deg - lo), v, lval);
                else
                  atomicCAS(&c->err, 0u, kDevErrQueue);
              }
            }
          }
        }
      }
      my_hbm = warp_sum(my_hbm);
      my_link = warp_sum(my_link);
      if (lane == 0 && my_hbm + my_link) {
        atomicAdd(&c->hbm_bytes, my_hbm);
        atomicAdd(&c->link_bytes, my_link);
      }
      if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
      // ------------------------------------------------------- expansion
      const unsigned long long ns = ldcg(&c->cnt_small[slot]);
      const unsigned long long nb = ldcg(&c->cnt_big[slot]);
      unsigned gsize = 32;
      while (gsize > 4 && nb + (ns + gsize - 1) / gsize < nwarps / 2) gsize >>= 1;
      const unsigned long long ngrp = (ns + gsize - 1) / gsize;
      const unsigned parts =
          nb && nb + ngrp < nwarps ? (unsigned)min(8ull, max(1ull, (nwarps - ngrp) / nb)) : 1u;
      const unsigned long long nbt = nb * parts, ntask = nbt + ngrp;
      // a level with few out-edges also lists the vertices it finds, so
      // that the next level can run in one CTA
      listed = a.flist && mf <= kLocalCap;
      NextLevel nl{N, 0, 0, listed ? a.flist + nslot * kLocalCap : nullptr, &c->fl_cnt[nslot]};
      for (unsigned long long t = gwarp; t < ntask;) {
        unsigned long long nt = 0;
        if (lane == 0) nt = atomicAdd(&c->wc[slot], 1ull);
        if (t < nbt) process_chunk<OP_BFS, ESZ, true>(a, a.qb[t / parts], (unsigned)(t % parts), parts, &nl);
        else process_group<OP_BFS, ESZ, true>(a, (t - nbt) * gsize, ns, gsize, &nl);
        t = nwarps + shfl64(nt, 0);
      }
      nl.nf = warp_sum(nl.nf);
      nl.mf = warp_sum(nl.mf);
      if (lane == 0 && nl.nf) {
        atomicAdd(&c->nf[nslot], nl.nf);
        atomicAdd(&c->mf[nslot], nl.mf);
      }
      if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
    }
    uint32_t *x = F;
    F = N;
    N = x;
  }
  if (leader) c->iters = iter;
}

template <int OP, int ESZ>
__global__ void __launch_bounds__(kMinThreads)
    minprop_kernel(MinArgs a) {
  // block table (first vertex, base address) in shared memory when it fits
  extern __shared__ unsigned long long s_tab[];
  __shared__ uint32_t s_word[kMinThreads / 32][64];  // compaction: taken bits, least kept value per word
  const bool smem_tab = a.nblk <= kSmemBlocks;
  unsigned long long *s_base = s_tab;
  uint32_t *s_vb = reinterpret_cast<uint32_t *>(s_tab + a.nblk);
  if (smem_tab) {
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];
    for (uint32_t i = threadIdx.x; i < a.nblk; i += blockDim.x) s_base[i] = a.blk_base[i];
  }
  __syncthreads();
  const uint32_t *vb = smem_tab ? s_vb : a.blk_vb;
  const unsigned long long *bbase = smem_tab ? s_base : (const unsigned long long *)a.blk_base;
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;

  // Only pending vertices with value < thr are expanded.  SSSP: a window of
  // fixed width above the smallest pending distance.  CC: labels in
  // increasing order, the window growing geometrically each time it empties,
  // so each component's minimum label floods it in one wave.
  uint32_t thr = 0xFFFFFFFFu;
  uint32_t width = a.delta;
  if (OP == OP_SSSP) thr = (uint32_t)min(1ull + a.delta, 0xFFFFFFFFull);
  if (OP == OP_CC) thr = a.delta;
  unsigned iter = 0;
  for (;; ++iter) {
    if (iter >= a.max_iters) {
      if (leader) atomicCAS(&c->err, 0u, kDevErrIters);
      break;
    }
    const unsigned slot = iter % 3, nslot = (iter + 1) % 3;
    if (leader) {
      c->cnt_small[nslot] = 0;
      c->cnt_big[nslot] = 0;
      c->cnt_host[nslot] = 0;
      c->remaining[nslot] = 0;
      c->wc[nslot] = 0;
      c->wc_host[nslot] = 0;
      c->minkept[nslot] = 0xFFFFFFFFu;
      c->mf[nslot] = 0;
      c->nf[nslot] = 0;
      c->bu_scan[nslot] = 0;
    }
    // ---------------------------------------------------------- compaction
    // A warp owns 32 bitmap words (lane = word).  The pending vertices of
    // its words are numbered across the warp and handled 32 per step (lane =
    // vertex), however they are spread over the words, so a group costs
    // ceil(pending / 32) steps instead of one step per non-empty word;
    // per-word results (taken bits, least kept value) gather in shared
    // memory and each word is rewritten once.  Queue items come out in
    // vertex order.
    unsigned long long my_edges = 0, my_hbm = 0, my_link = 0, my_verts = 0;
    unsigned long long my_keep = 0;
    uint32_t my_min = 0xFFFFFFFFu;
    uint32_t *s_tk = s_word[threadIdx.x >> 5], *s_km = s_tk + 32;
    // Fewer groups than warps (small graphs): BFS shares each group among
    // nsub warps, each taking every nsub-th step of the group's numbered
    // vertices.  BFS takes every pending vertex, so the group's words end
    // up empty; the last of its warps to finish (a per-group counter that
    // wraps back to 0) clears them, after every one of them has read them.
    const unsigned nsub =
        OP == OP_BFS && a.wmin && a.ngroups * 2u <= nwarps ? min(8u, nwarps / a.ngroups) : 1u;
    const unsigned gstride = nwarps / nsub, sub = gwarp % nsub;
    for (unsigned g = gwarp / nsub; g < a.ngroups && gwarp / nsub < gstride; g += gstride) {
      const unsigned wbase = g * 32u;
      const uint32_t word = ldcg(a.bm + wbase + lane);
      bool act_word = word != 0;
      if (OP != OP_BFS) {
        // a word whose pending values are all >= thr is kept without
        // touching its vertices
        const uint32_t wm = word ? ldcg(a.wmin + wbase + lane) : 0xFFFFFFFFu;
        if (word != 0 && wm >= thr) {
          my_keep += __popc(word);
          my_min = min(my_min, wm);
          act_word = false;
        }
      }
      const unsigned cnt = act_word ? (unsigned)__popc(word) : 0u;
      const unsigned incl = warp_incl_scan<unsigned>(cnt);
      const unsigned excl = incl - cnt, total = __shfl_sync(kFull, incl, 31);
      if (total == 0) continue;
      s_tk[lane] = 0;
      s_km[lane] = 0xFFFFFFFFu;
      __syncwarp();
      for (unsigned k = 32u * sub; k < total; k += 32u * nsub) {
        const unsigned t = k + lane;
        const int own = warp_owner(excl, t);
        const uint32_t ow = __shfl_sync(kFull, word, own);
        const unsigned oex = __shfl_sync(kFull, excl, own);
        const bool in = t < total;
        const uint32_t v = in ? (wbase + own) * 32u + nth_set_bit(ow, t - oex) : 0u;
        uint64_t s0 = 0, e0 = 0;
        // BFS takes every pending vertex: its offsets load beside its value
        if (OP == OP_BFS && in) {
          s0 = __ldg(a.off + v);
          e0 = __ldg(a.off + v + 1);
        }
        const uint32_t vval = in ? ldcg(a.val + v) : 0u;
        const bool take = in && (OP == OP_BFS || vval < thr);
        if (take) atomicOr(&s_tk[own], 1u << (v & 31u));
        else if (OP != OP_BFS && in) atomicMin(&s_km[own], vval);
        uint32_t deg = 0;
        unsigned long long eaddr = 0;
        bool host = false;
        if (take) {
          if (OP != OP_BFS) {
            s0 = __ldg(a.off + v);
            e0 = __ldg(a.off + v + 1);
          }
          deg = (uint32_t)(e0 - s0);
          const uint32_t bi = find_block(vb, a.nblk, v);
          eaddr = list_addr(a.lc, bbase[bi], a.host_base, v, s0, deg, ESZ, &host);
          if (a.blk_access) atomicAdd(a.blk_access + bi, (unsigned long long)deg * ESZ);
          my_edges += deg;
          my_verts += 1;
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
            if (pos < a.cap_s) a.qs[pos] = make_item(eaddr, deg, v, vval);
            else atomicCAS(&c->err, 0u, kDevErrQueue);
          }
        }
        // chunks of HBM lists fill the chunk queue from the bottom, chunks
        // of host-resident lists from the top (the link warps' pool; both
        // counts are checked against cap_b after the barrier)
        if (__any_sync(kFull, big)) {
          const unsigned nch = big ? (deg + a.chunk - 1) / a.chunk : 0u;
          const unsigned inc_r = warp_incl_scan<unsigned>(host ? 0u : nch);
          const unsigned inc_h = warp_incl_scan<unsigned>(host ? nch : 0u);
          const unsigned tot_r = __shfl_sync(kFull, inc_r, 31), tot_h = __shfl_sync(kFull, inc_h, 31);
          unsigned long long base = 0;
          if (lane == 0 && tot_r) base = atomicAdd(&c->cnt_big[slot], (unsigned long long)tot_r);
          if (lane == 1 && tot_h) base = atomicAdd(&c->cnt_host[slot], (unsigned long long)tot_h);
          const unsigned long long b_r = shfl64(base, 0), b_h = shfl64(base, 1);
          if (big) {
            unsigned long long pos = host ? b_h + inc_h - nch : b_r + inc_r - nch;
            for (unsigned kk = 0; kk < nch; kk++, pos++) {
              const uint32_t lo = kk * a.chunk;
              const uint32_t cn = min(a.chunk, deg - lo);
              if (pos < a.cap_b)
                a.qb[host ? a.cap_b - 1 - pos : pos] =
                    make_item(eaddr + (unsigned long long)lo * ESZ, cn, v, vval);
              else
                atomicCAS(&c->err, 0u, kDevErrQueue);
            }
          }
        }
      }
      __syncwarp();
      if (nsub > 1) {
        unsigned last = 0;
        if (lane == 0) last = atomicInc(a.wmin + g, nsub - 1u) == nsub - 1u;
        if (__shfl_sync(kFull, last, 0) && act_word) a.bm[wbase + lane] = 0;
      } else if (act_word) {
        const uint32_t tk = s_tk[lane];
        if (OP != OP_BFS) {
          const uint32_t km = s_km[lane];
          a.wmin[wbase + lane] = km;
          my_keep += __popc(word & ~tk);
          my_min = min(my_min, km);
        }
        if (tk) a.bm[wbase + lane] = word & ~tk;
      }
      __syncwarp();
    }
    my_edges = warp_sum(my_edges);
    my_hbm = warp_sum(my_hbm);
    my_link = warp_sum(my_link);
    my_verts = warp_sum(my_verts);
    if (OP != OP_BFS) {
      my_min = warp_min(my_min);
      my_keep = warp_sum(my_keep);
    }
    if (lane == 0 && my_verts) {
      // BFS edges are counted once the level's direction is known
      if (OP == OP_BFS) {
        atomicAdd(&c->mf[slot], my_edges);
        atomicAdd(&c->nf[slot], my_verts);
      } else {
        atomicAdd(&c->edges, my_edges);
      }
      atomicAdd(&c->hbm_bytes, my_hbm);
      atomicAdd(&c->link_bytes, my_link);
      atomicAdd(&c->vertices, my_verts);
    }
    if (OP != OP_BFS && lane == 0) {
      if (my_keep) atomicAdd(&c->remaining[slot], my_keep);
      if (my_min != 0xFFFFFFFFu) atomicMin(&c->minkept[slot], my_min);
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;

    const unsigned long long ns = ldcg(&c->cnt_small[slot]);
    const unsigned long long nb = ldcg(&c->cnt_big[slot]);
    const unsigned long long nh = ldcg(&c->cnt_host[slot]);
    if (nb + nh > a.cap_b) {  // the two ends of the chunk queue met
      if (leader) atomicCAS(&c->err, 0u, kDevErrQueue);
      break;
    }
    if (ns + nb + nh == 0) {
      if (OP == OP_BFS) break;
      if (ldcg(&c->remaining[slot]) == 0) break;
      const uint32_t mk = ldcg(&c->minkept[slot]);
      width = (uint32_t)min((unsigned long long)width * a.growth, 0xFFFFFFFFull);
      thr = (uint32_t)min((unsigned long long)mk + width, 0xFFFFFFFFull);
      continue;
    }
    if (OP == OP_BFS && leader) atomicAdd(&c->edges, ldcg(&c->mf[slot]));
    // ----------------------------------------------------------- expansion
    // task ids: chunks first, then groups of 32 small vertices; each warp
    // starts on task gwarp, then draws from a shared counter (no atomic at
    // all for warps without a first task)
    // With fewer tasks than warps, each chunk is split into up to 8 parts
    // (one task each) so that more warps share a small level's edges,
    // and groups of small vertices get smaller (down to 4 vertices)
    unsigned gsize = 32;
    const unsigned long long nchunks = nb + nh;
    while (gsize > 4 && nchunks + (ns + gsize - 1) / gsize < nwarps / 2) gsize >>= 1;
    const unsigned long long ngrp = (ns + gsize - 1) / gsize;
    const unsigned parts =
        nchunks && nchunks + ngrp < nwarps
            ? (unsigned)min(8ull, max(1ull, (nwarps - ngrp) / nchunks)) : 1u;
    const unsigned long long nbt = nb * parts, nht = nh * parts;
    const unsigned long long ntask = nbt + ngrp;
    // Two task pools, as in queue mode: one warp in link_every drains the
    // host-list chunks first (the link is busy from the phase's start), the
    // others take HBM chunks and groups first; each then helps with the
    // other pool.  First tasks are static, later ones come from the pool's
    // counter; a warp reserves its next task before working on this one.
    const unsigned le = a.link_every;
    const unsigned nlink = le ? (nwarps + le - 1) / le : 0u;
    const bool link_warp = le && gwarp % le == 0;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
      const bool hpool = link_warp == (pass == 0);
      unsigned long long *ctr = hpool ? &c->wc_host[slot] : &c->wc[slot];
      const unsigned long long n = hpool ? nht : ntask;
      const unsigned long long first = hpool ? nlink : nwarps - nlink;
      unsigned long long t;
      if (pass == 0) {
        t = link_warp ? gwarp / le : gwarp - (le ? gwarp / le + 1 : 0u);
      } else {
        unsigned long long f = 0;
        if (lane == 0 && first < n) f = atomicAdd(ctr, 1ull);
        t = first + shfl64(f, 0);
      }
      while (t < n) {
        unsigned long long nt = 0;
        if (lane == 0) nt = atomicAdd(ctr, 1ull);
        if (hpool) {
          const MinItem it = a.qb[a.cap_b - 1 - t / parts];
          process_chunk<OP, ESZ>(a, it, (unsigned)(t % parts), parts);
        } else if (t < nbt) {
          const MinItem it = a.qb[t / parts];
          process_chunk<OP, ESZ>(a, it, (unsigned)(t % parts), parts);
        } else {
          process_group<OP, ESZ>(a, (t - nbt) * gsize, ns, gsize);
        }
        t = first + shfl64(nt, 0);
      }
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
  }
  if (leader) c->iters = iter;
}

template <int OP>
__global__ void minprop_init(MinArgs a, uint32_t nw_alloc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t v = tid; v < a.nv; v += stride)
    a.val[v] = OP == OP_CC ? (uint32_t)v : (v == a.src ? 1u : a.nv + 1u);
  for (uint64_t w = tid; w < nw_alloc; w += stride) {
    uint32_t word = 0;
    if (OP == OP_CC) {
      // every vertex with out-edges is pending with its own id as label
      const uint64_t lo = w * 32ull;
      const uint64_t hi = lo + 32ull < (uint64_t)a.nv ? lo + 32ull : (uint64_t)a.nv;
      uint64_t prev = lo < hi ? a.off[lo] : 0;
      for (uint64_t v = lo; v < hi; v++) {
        const uint64_t nx = a.off[v + 1];
        if (nx > prev) word |= 1u << (v - lo);
        prev = nx;
      }
      a.wmin[w] = lo < 0xFFFFFFFFull ? (uint32_t)lo : 0xFFFFFFFFu;
    } else if (w == (a.src >> 5)) {
      word = 1u << (a.src & 31u);
    }
    a.bm[w] = word;
    if (OP == OP_SSSP) a.wmin[w] = w == (a.src >> 5) ? 1u : 0xFFFFFFFFu;
    // BFS: per-group counters of the warps that share a compaction group,
    // and the second frontier bitmap of direction-optimising runs
    if (OP == OP_BFS && a.wmin) a.wmin[w] = 0;
    if (OP == OP_BFS && a.bm2) a.bm2[w] = 0;
  }
  if (tid == 0) {
    MinCtrl *c = a.ctrl;
    memset(c, 0, sizeof(MinCtrl));
    for (int s = 0; s < 3; s++) c->minkept[s] = 0xFFFFFFFFu;
  }
}

// ================================================================ queue mode
//
// Same relaxation and windows as minprop_kernel, but a relaxation that
// lowers a vertex below the window pushes it straight into the next
// iteration's queue (degree, block and warp-aggregated append done by the
// pusher), so an iteration is one expansion phase and one grid barrier.
// The bitmap scan runs only when the near queue is empty: at the start, and
// when an SSSP/CC window advances over vertices parked in the far bitmap.
//
// SSSP/CC push a vertex at most once per queue through two bitmaps of
// queued vertices, one per phase parity (one bit per vertex: small enough
// to stay in L2 beside the values, which per-vertex 4-byte tags were not).
// A relaxation in phase ph that lowers w below the window pushes it only if
// its atomicOr on w's bit in Q[ph & 1] found the bit clear.  Invariant: w's
// bit in Q[ph & 1] set implies w has an entry in phase ph's output queue,
// which phase ph + 1 expands after a grid barrier and so with the final
// value of phase ph.  The expander of phase ph + 1 clears the bit of every
// entry it takes in Q[ph & 1] (so Q[ph & 1] is empty again when phase ph + 2
// pushes into it) and skips an entry whose bit in Q[(ph + 1) & 1] is already
// set (it is queued again, with a lower value); otherwise it expands with
// the value it reads.  No decrease is lost under any ordering of the two
// sides, so no fence is needed; a late bit read only costs a redundant
// expansion.  Entries queued by a bitmap scan have no bit (the scan takes
// each vertex once).  BFS needs neither: a vertex changes once and its
// pusher is unique.

// Expansion accounting, per warp in shared memory (registers are the
// queue-mode kernel's limit): edges expanded and their bytes by where they
// live.  Only lane 0 updates it.
struct QStats {
  unsigned long long *s;  // [0] edges, [1] HBM bytes, [2] link bytes
};

__device__ __forceinline__ void q_count(const MinArgs &a, QStats &qst, unsigned long long eaddr,
                                        unsigned cnt, unsigned esz) {
  qst.s[0] += cnt;
  const unsigned long long b = (unsigned long long)cnt * esz;
  if (eaddr >= a.host_base && eaddr < a.host_end) qst.s[2] += b;  // cache lies outside
  else qst.s[1] += b;
}

// Warp-uniform: lanes with `flag` append vertex w (value wval) to the queue
// pair (qs, qb) whose counters live in slot cs.
template <int ESZ>
__device__ __forceinline__ void q_append(const MinArgs &a, const uint32_t *vb,
                                         const unsigned long long *bbase, MinItem *qs,
                                         MinItem *qb, unsigned cs, bool flag, uint32_t w,
                                         uint32_t wval, QStats &qst) {
  if (!__any_sync(kFull, flag)) return;
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  uint32_t deg = 0;
  unsigned long long eaddr = 0;
  bool host = false;
  if (flag) {
    // the block (shared memory) and, for a host block, the small-list
    // cache slot depend on w alone: that load travels with the offsets'
    const uint32_t bi = find_block(vb, a.nblk, w);
    const unsigned long long bb = bbase[bi];
    const bool host_blk = bb == a.host_base;
    const uint32_t slot = host_blk && a.lc.deg_lt ? __ldg(a.lc.idx + w) : 0u;
    const uint64_t s0 = __ldg(a.off + w), e0 = __ldg(a.off + w + 1);
    deg = (uint32_t)(e0 - s0);
    if (host_blk && deg > 0 && deg < a.lc.deg_lt) {
      eaddr = a.lc.base + (unsigned long long)slot * ESZ;
    } else {
      host = host_blk;
      eaddr = bb + s0 * ESZ;
    }
    if (a.blk_access) atomicAdd(a.blk_access + bi, (unsigned long long)deg * ESZ);
  }
  // Lists read over the host link always go to chunk items (whole-line
  // loads by the link warps); the small-vertex groups take only lists in
  // HBM (resident blocks, small-list cache), whose scattered 4-byte loads
  // would waste most of each host-link request.
  const bool small = flag && deg > 0 && deg < a.small_deg && !host;
  const bool big = flag && deg > 0 && !small;
  // Chunks of HBM lists fill the chunk queue from the bottom, chunks of
  // host-resident lists from the top (the expansion hands them to the
  // link warps first); the two counts together stay within cap_b, which
  // every block checks after the phase's barrier, before any item is read.
  // The three reservations (small items, HBM chunks, host chunks) go out
  // together from lanes 0, 1 and 2.
  const unsigned sm = __ballot_sync(kFull, small);
  const unsigned nch = big ? (deg + a.chunk - 1) / a.chunk : 0u;
  const unsigned inc_r = warp_incl_scan<unsigned>(host ? 0u : nch);
  const unsigned inc_h = warp_incl_scan<unsigned>(host ? nch : 0u);
  const unsigned tot_r = __shfl_sync(kFull, inc_r, 31), tot_h = __shfl_sync(kFull, inc_h, 31);
  unsigned long long base = 0;
  if (lane == 0 && sm) base = atomicAdd(&c->cnt_small[cs], (unsigned long long)__popc(sm));
  if (lane == 1 && tot_r) base = atomicAdd(&c->cnt_big[cs], (unsigned long long)tot_r);
  if (lane == 2 && tot_h) base = atomicAdd(&c->cnt_host[cs], (unsigned long long)tot_h);
  const unsigned long long b_s = shfl64(base, 0), b_r = shfl64(base, 1), b_h = shfl64(base, 2);
  if (small) {
    const unsigned long long pos = b_s + __popc(sm & lanemask_lt());
    if (pos < a.cap_s) qs[pos] = make_item(eaddr, deg, w, wval);
    else atomicCAS(&c->err, 0u, kDevErrQueue);
  }
  if (big) {
    unsigned long long pos = host ? b_h + inc_h - nch : b_r + inc_r - nch;
    for (unsigned k = 0; k < nch; k++, pos++) {
      const uint32_t lo = k * a.chunk;
      if (pos < a.cap_b)
        qb[host ? a.cap_b - 1 - pos : pos] =
            make_item(eaddr + (unsigned long long)lo * ESZ, min(a.chunk, deg - lo), w, wval);
      else
        atomicCAS(&c->err, 0u, kDevErrQueue);
    }
  }
}

struct QEnv {
  const uint32_t *vb;
  const unsigned long long *bbase;
  MinItem *qs_next, *qb_next;
  unsigned cs_next;
  uint32_t thr;
  uint32_t *qnext;  // queued bits of this phase's output queue
  uint32_t *qprev;  // queued bits of the queue this phase expands
  uint2 *stage;  // this warp's shared list of vertices to queue: (w, value)
};

// Queue-mode relaxation: up to this many edges per lane in one call.
constexpr int kQRelaxMax = 8;
// Queue-mode scan: pending vertices probed per lane per step.
constexpr int kScanPer = 4;
// Queue-mode small-vertex groups: edges per lane per step (2 and 4
// measured slower at RMAT-24).
constexpr int kGroupPer = 8;

// Appends the warp's staged vertices in batches of 32 lanes.  Unless all is
// set, only whole batches go and the rest (fewer than 32) moves to the front
// of the list, so a warp appends once per 32 queued vertices, however few
// each relaxation step queues.  A vertex's queued bit is set when it is
// staged; every staged vertex is appended before the phase's closing
// barrier (the final call with all = true), so the bit still implies an
// entry in this phase's queue.
template <int ESZ>
__device__ __forceinline__ void q_flush(const MinArgs &a, const QEnv &e, unsigned &nst, bool all,
                                        QStats &qst) {
  const unsigned lane = lane_id();
  const unsigned take = all ? nst : (nst & ~31u);
  if (!take) return;
  __syncwarp();
  for (unsigned k = 0; k < take; k += 32) {
    const bool f = k + lane < take;
    const uint2 x = f ? e.stage[k + lane] : make_uint2(0, 0);
    q_append<ESZ>(a, e.vb, e.bbase, e.qs_next, e.qb_next, e.cs_next, f, x.x, x.y, qst);
  }
  const unsigned rest = nst - take;
  const uint2 x = lane < rest ? e.stage[take + lane] : make_uint2(0, 0);
  __syncwarp();
  if (lane < rest) e.stage[lane] = x;
  __syncwarp();
  nst = rest;
}

// Relax N edges per lane; near improvements are queued, far ones parked.
// Each dependent step (value probe, atomicMin, queued-bit claim) is issued
// for all N edges before any result is used, so a lane has N requests in
// flight per step instead of one.  The vertices to queue are staged in the
// warp's shared list (nst entries, warp-uniform) and appended 32 at a time
// by q_flush.  cand is the saturated u32 candidate (0xFFFFFFFF never wins).
template <int OP, int ESZ, int N>
__device__ __forceinline__ void q_relax_n(const MinArgs &a, const QEnv &e, const uint32_t (&w)[N],
                                          const uint32_t (&cand)[N], const bool (&ok)[N],
                                          unsigned &nst, QStats &qst) {
  static_assert(N <= kQRelaxMax, "one step stages at most kQRelaxMax entries per lane");
  // values stay in L2 (evict-last) while edges and items stream through
  const unsigned long long keep = l2_evict_last();
  uint32_t r[N];
#pragma unroll
  for (int j = 0; j < N; j++) r[j] = ok[j] ? ldcg_hint(a.val + w[j], keep) : 0u;
  bool push[N];
  if (OP == OP_BFS) {
    // the discoverer is the one whose atomicMin lowered the value
#pragma unroll
    for (int j = 0; j < N; j++)
      r[j] = ok[j] && cand[j] < r[j] ? atomic_min_hint(a.val + w[j], cand[j], keep) : 0u;
#pragma unroll
    for (int j = 0; j < N; j++) push[j] = cand[j] < r[j];  // 0 when not attempted
  } else {
    // SSSP/CC: an edge whose candidate beats the probed value lowers it
    // fire-and-forget, and a near one claims w's queued bit in the same
    // round trip, before the atomicMin's outcome is known: a claim that
    // finds the bit clear pushes w even if a concurrent relaxation lowered
    // val[w] below the candidate first.  Then that relaxation (also near:
    // its candidate is smaller) finds the bit set and does not push, so w
    // is queued exactly once either way, and the expansion reads the
    // current value.  A far candidate parks w fire-and-forget; parking
    // after such a race only loosens the word's lower bound.
#pragma unroll
    for (int j = 0; j < N; j++) {
      const bool att = ok[j] && cand[j] < r[j];
      const bool near = att && cand[j] < e.thr;
      r[j] = near ? atomicOr(e.qnext + (w[j] >> 5), 1u << (w[j] & 31u)) : 0xFFFFFFFFu;
      if (att) red_min_hint(a.val + w[j], cand[j], keep);
      if (att && !near) {
        atomicMin(a.wmin + (w[j] >> 5), cand[j]);
        atomicOr(a.bm + (w[j] >> 5), 1u << (w[j] & 31u));
      }
    }
#pragma unroll
    for (int j = 0; j < N; j++) push[j] = !((r[j] >> (w[j] & 31u)) & 1u);
  }
#pragma unroll
  for (int j = 0; j < N; j++) {
    const unsigned b = __ballot_sync(kFull, push[j]);
    if (push[j]) e.stage[nst + __popc(b & lanemask_lt())] = make_uint2(w[j], cand[j]);
    nst += __popc(b);
  }
  if (nst >= 32) q_flush<ESZ>(a, e, nst, false, qst);
}

// Dequeue: BFS values are final when queued.  SSSP/CC clear the vertex's
// parked bit (its pending value is handled here) and its queued bit of this
// queue, read the latest value and report a skip when the vertex is already
// queued again for the next phase.
template <int OP>
__device__ __forceinline__ uint32_t q_dequeue(const MinArgs &a, const QEnv &e, uint32_t v,
                                              uint32_t item_val, bool &skip) {
  skip = false;
  if (OP == OP_BFS) return item_val;
  const uint32_t m = 1u << (v & 31u);
  if (ldcg(a.bm + (v >> 5)) & m) atomicAnd(a.bm + (v >> 5), ~m);
  atomicAnd(e.qprev + (v >> 5), ~m);
  const uint32_t cur = ldcg_hint(a.val + v, l2_evict_last());
  skip = (ldcg(e.qnext + (v >> 5)) & m) != 0;
  return cur;
}

template <int OP, int ESZ>
__device__ __forceinline__ void q_chunk(const MinArgs &a, const QEnv &e, const MinItem &it,
                                        unsigned part, unsigned parts, unsigned &nst,
                                        QStats &qst) {
  constexpr int PER = 16 / ESZ;
  const unsigned lane = lane_id();
  // part `part` of `parts` of the chunk (whole 32-edge runs): small phases
  // split their chunks so that more warps share them
  const uint32_t cnt = (uint32_t)(it.ea_cnt >> 48);
  const uint32_t per = ((cnt + parts - 1) / parts + 31u) & ~31u;
  const uint32_t lo = min(cnt, part * per), hi = min(cnt, lo + per);
  if (lo >= hi) return;
  const uintptr_t start = (it.ea_cnt & kAddrMask) + (uintptr_t)lo * ESZ;
  const uintptr_t end = (it.ea_cnt & kAddrMask) + (uintptr_t)hi * ESZ;
  // two 16-byte loads per lane in flight (1 KiB per warp step): host-link
  // reads are latency-bound per warp.  The next step's loads are issued
  // before this step's relaxation, so they travel while its probes and
  // atomics do.  An HBM chunk's first loads also go out before the
  // dequeue's, which they do not depend on (a skipped item wastes 1 KiB of
  // HBM reads); a host chunk's wait for the dequeue, so that skipped items
  // cost no link bytes.
  // edges are read once: evict-first
  const unsigned long long stream = l2_evict_first();
  const bool on_link = start >= a.host_base && start < a.host_end;
  uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane;
  uint4 qn[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
  if (!on_link) {
#pragma unroll
    for (int h = 0; h < 2; h++)
      if (p + 512u * h < end) qn[h] = ld_stream_v4(p + 512u * h, stream);
  }
  uint32_t vval = it.val;
  if (OP != OP_BFS) {
    bool skip = false;
    if (lane == 0) vval = q_dequeue<OP>(a, e, it.v, it.val, skip);
    vval = __shfl_sync(kFull, vval, 0);
    if (__shfl_sync(kFull, skip, 0)) return;
  }
  if (lane == 0) q_count(a, qst, start, hi - lo, ESZ);
  if (on_link) {
#pragma unroll
    for (int h = 0; h < 2; h++)
      if (p + 512u * h < end) qn[h] = ld_stream_v4(p + 512u * h, stream);
  }
  for (; __any_sync(kFull, p < end); p += 1024u) {
    uint4 q[2] = {qn[0], qn[1]};
#pragma unroll
    for (int h = 0; h < 2; h++)
      qn[h] = p + 1024u + 512u * h < end ? ld_stream_v4(p + 1024u + 512u * h, stream)
                                          : make_uint4(0, 0, 0, 0);
    uint32_t w[2 * PER], cand[2 * PER];
    bool ok[2 * PER];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint32_t f[4] = {q[h].x, q[h].y, q[h].z, q[h].w};
#pragma unroll
      for (int j = 0; j < PER; j++) {
        const uintptr_t ea = p + 512u * h + (uintptr_t)ESZ * j;
        const int k = h * PER + j;
        ok[k] = ea >= start && ea < end;
        w[k] = ESZ == 4 ? edge_dst(f[j], a.wshift) : f[2 * j];
        cand[k] = sat32(candidate<OP>(vval, ESZ == 4 ? edge_wt(f[j], a.wshift, a.wbase) : f[2 * j + 1]));
      }
    }
    q_relax_n<OP, ESZ, 2 * PER>(a, e, w, cand, ok, nst, qst);
  }
}

template <int OP, int ESZ>
__device__ __forceinline__ void q_group(const MinArgs &a, const QEnv &e, const MinItem *qs,
                                        unsigned long long first, unsigned long long n_small,
                                        unsigned gsize, unsigned &nst, QStats &qst) {
  const unsigned lane = lane_id();
  const unsigned long long idx = first + lane;
  MinItem it{0, 0, 0};
  const bool valid = lane < gsize && idx < n_small;
  if (valid) it = qs[idx];
  bool skip = !valid;
  uint32_t vval = 0;
  if (valid) vval = q_dequeue<OP>(a, e, it.v, it.val, skip);
  const unsigned cnt = skip ? 0u : (unsigned)(it.ea_cnt >> 48);
  const unsigned long long eaddr = it.ea_cnt & kAddrMask;
  {
    // the group's edges and link bytes, summed over the lanes
    const bool on_link = eaddr >= a.host_base && eaddr < a.host_end;
    const unsigned e_sum = __reduce_add_sync(kFull, cnt);
    const unsigned l_sum = __reduce_add_sync(kFull, on_link ? cnt : 0u);
    if (lane == 0 && e_sum) {
      qst.s[0] += e_sum;
      qst.s[1] += (unsigned long long)(e_sum - l_sum) * ESZ;
      qst.s[2] += (unsigned long long)l_sum * ESZ;
    }
  }
  const unsigned incl = warp_incl_scan<unsigned>(cnt);
  const unsigned excl = incl - cnt;
  const unsigned total = __shfl_sync(kFull, incl, 31);
  // kGroupPer x 32 edges per step, kGroupPer per lane in flight
  for (unsigned k = 0; k < total; k += 32u * kGroupPer) {
    uint32_t w[kGroupPer], cand[kGroupPer];
    bool ok[kGroupPer];
#pragma unroll
    for (int h = 0; h < kGroupPer; h++) {
      w[h] = 0;
      const unsigned t = k + 32u * h + lane;
      const int o = warp_owner(excl, t);
      const unsigned long long ea = shfl64(eaddr, o);
      const unsigned oex = __shfl_sync(kFull, excl, o);
      const uint32_t ov = __shfl_sync(kFull, vval, o);
      ok[h] = t < total;
      uint32_t wt = 0;
      if (ok[h]) {
        const uintptr_t addr = (uintptr_t)ea + (uintptr_t)(t - oex) * ESZ;
        if (ESZ == 4) {
          const uint32_t ed = ld_stream_u32(addr, l2_evict_first());
          w[h] = edge_dst(ed, a.wshift);
          wt = edge_wt(ed, a.wshift, a.wbase);
        } else {
          const uint2 ed = ld_stream_u2(addr, l2_evict_first());
          w[h] = ed.x;
          wt = ed.y;
        }
      }
      cand[h] = sat32(candidate<OP>(ov, wt));
    }
    q_relax_n<OP, ESZ, kGroupPer>(a, e, w, cand, ok, nst, qst);
  }
}

template <int OP, int ESZ>
// Two blocks per SM: 64 registers, no spills (3 blocks spill and measured slower).
__global__ void __launch_bounds__(kMinThreads, 2) minq_kernel(MinArgs a) {
  extern __shared__ unsigned long long s_tab[];
  // staging list: fewer than 32 carried entries plus one relaxation step's
  __shared__ uint2 s_stage[kMinThreads / 32][32 * (kQRelaxMax + 1)];
  __shared__ uint32_t s_word[kMinThreads / 32][64];  // scan: taken bits, least kept value per word
  const bool smem_tab = a.nblk <= kSmemBlocks;
  unsigned long long *s_base = s_tab;
  uint32_t *s_vb = reinterpret_cast<uint32_t *>(s_tab + a.nblk);
  if (smem_tab) {
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];
    for (uint32_t i = threadIdx.x; i < a.nblk; i += blockDim.x) s_base[i] = a.blk_base[i];
  }
  __syncthreads();
  QEnv env;
  env.vb = smem_tab ? s_vb : a.blk_vb;
  env.bbase = smem_tab ? s_base : (const unsigned long long *)a.blk_base;
  env.stage = s_stage[threadIdx.x >> 5];
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  uint32_t thr = 0xFFFFFFFFu;
  uint32_t width = a.delta;
  if (OP == OP_SSSP) thr = (uint32_t)min(1ull + a.delta, 0xFFFFFFFFull);
  if (OP == OP_CC) thr = a.delta;
  __shared__ unsigned long long s_qst[kMinThreads / 32][3];
  QStats qst{s_qst[threadIdx.x >> 5]};
  if (lane < 3) qst.s[lane] = 0;
  __syncwarp();
  // Every phase (scan or expansion) ph produces the queue in counter slot
  // ph % 3 and buffer ph & 1; an expansion consumes what phase ph - 1
  // produced.  The decision after a phase reads only that phase's slot,
  // which no block writes again before everyone has passed the next
  // barrier; the leader clears slot (ph + 1) % 3 at the start of phase ph.
  unsigned ph = 0, iter = 0;
  bool scan = true;
  for (;; ++iter, ++ph) {
    if (iter >= a.max_iters) {
      if (leader) atomicCAS(&c->err, 0u, kDevErrIters);
      break;
    }
    const unsigned cur = ph % 3, prev = (ph + 2) % 3;
    if (leader) {
      const unsigned r = (ph + 1) % 3;
      c->cnt_small[r] = 0;
      c->cnt_big[r] = 0;
      c->cnt_host[r] = 0;
      c->wc[r] = 0;
      c->wc_host[r] = 0;
      c->remaining[r] = 0;
      c->minkept[r] = 0xFFFFFFFFu;
    }
    MinItem *qs_out = (ph & 1) ? a.qs2 : a.qs, *qb_out = (ph & 1) ? a.qb2 : a.qb;
    MinItem *qs_in = (ph & 1) ? a.qs : a.qs2, *qb_in = (ph & 1) ? a.qb : a.qb2;
    env.qs_next = qs_out;
    env.qb_next = qb_out;
    env.cs_next = cur;
    env.thr = thr;
    env.qnext = a.qbits + (size_t)(ph & 1u) * a.ngroups * 32u;
    env.qprev = a.qbits + (size_t)((ph + 1u) & 1u) * a.ngroups * 32u;
    if (scan) {
      // ------------------------------------------------------------- scan
      // A warp owns 32 bitmap words (lane = word).  The pending vertices of
      // the words inside the window are numbered across the warp and probed
      // kScanPer x 32 at a time (independent loads, however sparse the
      // words); per-word results gather in shared memory (taken bits, least
      // kept value) and the words are rewritten once at the end.
      unsigned long long my_keep = 0;
      uint32_t my_min = 0xFFFFFFFFu;
      uint32_t *s_tk = s_word[threadIdx.x >> 5], *s_km = s_tk + 32;
      unsigned nst = 0;  // vertices staged in this warp's list, not yet appended
      for (unsigned g = gwarp; g < a.ngroups; g += nwarps) {
        const unsigned wbase = g * 32u;
        const uint32_t word = ldcg(a.bm + wbase + lane);
        bool act_word = word != 0;
        if (OP != OP_BFS) {
          const uint32_t wm = word ? ldcg(a.wmin + wbase + lane) : 0xFFFFFFFFu;
          if (word != 0 && wm >= thr) {
            my_keep += __popc(word);
            my_min = min(my_min, wm);
            act_word = false;
          }
        }
        const unsigned cnt = act_word ? (unsigned)__popc(word) : 0u;
        const unsigned incl = warp_incl_scan<unsigned>(cnt);
        const unsigned excl = incl - cnt, total = __shfl_sync(kFull, incl, 31);
        if (total == 0) continue;
        s_tk[lane] = 0;
        s_km[lane] = 0xFFFFFFFFu;
        __syncwarp();
        for (unsigned k = 0; k < total; k += 32u * kScanPer) {
          uint32_t v[kScanPer], vv[kScanPer];
          int own[kScanPer];
#pragma unroll
          for (int i = 0; i < kScanPer; i++) {
            const unsigned t = k + 32u * i + lane;
            own[i] = warp_owner(excl, t);
            const uint32_t ow = __shfl_sync(kFull, word, own[i]);
            const unsigned oex = __shfl_sync(kFull, excl, own[i]);
            v[i] = t < total ? (wbase + own[i]) * 32u + nth_set_bit(ow, t - oex) : 0xFFFFFFFFu;
          }
#pragma unroll
          for (int i = 0; i < kScanPer; i++) vv[i] = v[i] != 0xFFFFFFFFu ? ldcg(a.val + v[i]) : 0u;
#pragma unroll
          for (int i = 0; i < kScanPer; i++) {
            const bool in = v[i] != 0xFFFFFFFFu;
            const bool take = in && (OP == OP_BFS || vv[i] < thr);
            if (take) atomicOr(&s_tk[own[i]], 1u << (v[i] & 31u));
            else if (OP != OP_BFS && in) atomicMin(&s_km[own[i]], vv[i]);
            const unsigned b = __ballot_sync(kFull, take);
            if (take) env.stage[nst + __popc(b & lanemask_lt())] = make_uint2(v[i], vv[i]);
            nst += __popc(b);
          }
          if (nst >= 32) q_flush<ESZ>(a, env, nst, false, qst);
          __syncwarp();
        }
        if (act_word) {
          const uint32_t tk = s_tk[lane];
          if (OP != OP_BFS) {
            const uint32_t km = s_km[lane];
            a.wmin[wbase + lane] = km;
            my_keep += __popc(word & ~tk);
            my_min = min(my_min, km);
          }
          if (tk) a.bm[wbase + lane] = word & ~tk;
        }
        __syncwarp();
      }
      q_flush<ESZ>(a, env, nst, true, qst);
      if (OP != OP_BFS) {
        my_keep = warp_sum(my_keep);
        my_min = warp_min(my_min);
        if (lane == 0) {
          if (my_keep) atomicAdd(&c->remaining[cur], my_keep);
          if (my_min != 0xFFFFFFFFu) atomicMin(&c->minkept[cur], my_min);
        }
      }
    } else {
      // --------------------------------------------------------- expansion
      // Two task pools: chunks of host-resident lists (read over the
      // link), and the rest (HBM chunks, then groups of small vertices).
      // One warp in link_every (the link warps) drains the host pool
      // first, so the link is busy from the phase's start while the other
      // warps work through HBM-resident lists; each warp then helps with
      // the other pool.  The first task of a warp's first pool is static
      // (its index among that pool's warps), the rest come from the pool's
      // counter.
      const unsigned long long ns = ldcg(&c->cnt_small[prev]);
      const unsigned long long nb = ldcg(&c->cnt_big[prev]);
      const unsigned long long nh = ldcg(&c->cnt_host[prev]);
      // With fewer tasks than warps (the small phases at a window's start
      // and end), groups shrink down to 4 vertices and each chunk is split
      // into up to 8 parts, so that more warps share the phase's edges.
      const unsigned long long nchunks = nb + nh;
      unsigned gsize = 32;
      while (gsize > 4 && nchunks + (ns + gsize - 1) / gsize < nwarps / 2) gsize >>= 1;
      const unsigned long long ngrp = (ns + gsize - 1) / gsize;
      const unsigned parts =
          nchunks && nchunks + ngrp < nwarps
              ? (unsigned)min(8ull, max(1ull, (nwarps - ngrp) / nchunks)) : 1u;
      const unsigned long long nbt = nb * parts, nht = nh * parts;
      const unsigned long long ntask = nbt + ngrp;
      const unsigned le = a.link_every;
      const unsigned nlink = le ? (nwarps + le - 1) / le : 0u;
      const bool link_warp = le && gwarp % le == 0;
      unsigned nst = 0;  // vertices staged in this warp's list, not yet appended
#pragma unroll 1
      for (int pass = 0; pass < 2; pass++) {
        const bool hpool = link_warp == (pass == 0);
        unsigned long long *ctr = hpool ? &c->wc_host[prev] : &c->wc[prev];
        const unsigned long long n = hpool ? nht : ntask;
        const unsigned long long first = hpool ? nlink : nwarps - nlink;
        unsigned long long t;
        if (pass == 0) {
          t = link_warp ? gwarp / le : gwarp - (le ? gwarp / le + 1 : 0u);
        } else {
          unsigned long long f = 0;
          if (lane == 0 && first < n) f = atomicAdd(ctr, 1ull);
          t = first + shfl64(f, 0);
        }
        while (t < n) {
          unsigned long long nt = 0;
          if (lane == 0) nt = atomicAdd(ctr, 1ull);
          if (hpool) {
            const MinItem it = qb_in[a.cap_b - 1 - t / parts];
            q_chunk<OP, ESZ>(a, env, it, (unsigned)(t % parts), parts, nst, qst);
          } else if (t < nbt) {
            const MinItem it = qb_in[t / parts];
            q_chunk<OP, ESZ>(a, env, it, (unsigned)(t % parts), parts, nst, qst);
          } else {
            q_group<OP, ESZ>(a, env, qs_in, (t - nbt) * gsize, ns, gsize, nst, qst);
          }
          t = first + shfl64(nt, 0);
        }
      }
      q_flush<ESZ>(a, env, nst, true, qst);
    }
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
    const unsigned long long nbig = ldcg(&c->cnt_big[cur]), nhost = ldcg(&c->cnt_host[cur]);
    if (nbig + nhost > a.cap_b) {  // the two ends of the chunk queue met
      if (leader) atomicCAS(&c->err, 0u, kDevErrQueue);
      break;
    }
    const unsigned long long produced = ldcg(&c->cnt_small[cur]) + nbig + nhost;
    if (produced) {
      scan = false;  // expand what this phase queued
    } else if (!scan) {
      scan = true;   // near queue empty: look at the parked vertices
    } else {
      if (OP == OP_BFS || ldcg(&c->remaining[cur]) == 0) break;
      const uint32_t mk = ldcg(&c->minkept[cur]);
      width = (uint32_t)min((unsigned long long)width * a.growth, 0xFFFFFFFFull);
      thr = (uint32_t)min((unsigned long long)mk + width, 0xFFFFFFFFull);
    }
  }
  __syncwarp();
  if (lane == 0 && qst.s[0]) {
    atomicAdd(&c->edges, qst.s[0]);
    atomicAdd(&c->hbm_bytes, qst.s[1]);
    atomicAdd(&c->link_bytes, qst.s[2]);
  }
  if (leader) c->iters = iter;
}

__global__ void minq_clear(uint32_t *qbits, uint32_t nwords) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += gridDim.x * blockDim.x)
    qbits[i] = 0;
}

__global__ void values_checksum_kernel(const uint32_t *val, uint64_t nv,
                                       unsigned long long *sum) {
  __shared__ unsigned long long s_red[32];
  unsigned long long h = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    unsigned long long x = (v << 32) | val[v];
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    h += x ^ (x >> 31);
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

// ============================================= union-find CC (symmetric)
//
// On a symmetric graph the min-label fixed point is the smallest id of each
// connected component, which union-find reaches without reading most of the
// adjacency (the sampling scheme of Afforest, Sutton et al., IPDPS'18):
//   1. every vertex unions with its first kUfSample neighbours;
//   2. flatten; c = the component of the highest-degree vertex;
//   3. every vertex outside c unions with the rest of its list; vertices in
//      c skip theirs -- an edge with both ends in c changes nothing, and an
//      edge with one end outside c is read from that end (its reverse is in
//      the other end's list);
//   4. flatten.
// Roots are hooked larger-under-smaller with a CAS, so a parent id never
// exceeds its child's and each root is its component's minimum id; finds
// shortcut the path as they climb.

__device__ __forceinline__ uint32_t uf_find(uint32_t *p, uint32_t x) {
  uint32_t cur = ldcg(p + x);
  if (cur == x) return x;
  uint32_t prev = x, next;
  while (cur > (next = ldcg(p + cur))) {
    p[prev] = next;  // shortcut to an ancestor: benign under races
    prev = cur;
    cur = next;
  }
  return cur;
}

__device__ __forceinline__ void uf_union(uint32_t *p, uint32_t u, uint32_t w) {
  uint32_t ru = uf_find(p, u), rw = uf_find(p, w);
  while (ru != rw) {
    const uint32_t hi = max(ru, rw), lo = min(ru, rw);
    const uint32_t old = atomicCAS(p + hi, hi, lo);
    if (old == hi) return;  // hooked
    // hi stopped being a root meanwhile: continue from the current roots
    ru = uf_find(p, old);
    rw = uf_find(p, lo);
  }
}

constexpr uint32_t kUfSample = 2;

// Step 1: each vertex (one thread) unions with its first kUfSample
// neighbours.  (Storing the smallest neighbour as the parent outright, with
// no CAS, measured slower: the parent chains it builds are long, and every
// later find climbs them.)
template <int ESZ>
__device__ __forceinline__ void uf_sample_edges(const MinArgs &a, const uint32_t *vb,
                                                const unsigned long long *bbase, uint32_t v,
                                                uint32_t (&w)[kUfSample], uint32_t &k, bool &host) {
  const uint64_t s = __ldg(a.off + v), e = __ldg(a.off + v + 1);
  const uint32_t deg = (uint32_t)(e - s);
  k = min(deg, kUfSample);
  host = false;
  if (!k) return;
  const unsigned long long eaddr =
      list_addr(a.lc, bbase[find_block(vb, a.nblk, v)], a.host_base, v, s, deg, ESZ, &host);
#pragma unroll
  for (uint32_t j = 0; j < kUfSample; j++) {
    const uint32_t raw = j < k ? ld_nc_u32(eaddr + (unsigned long long)j * ESZ) : v;
    w[j] = ESZ == 4 ? edge_dst(raw, a.wshift) : raw;
  }
}

// block table of the plan in shared memory (as minprop_kernel stages it)
#define UF_STAGE_BLOCKS()                                                                        \
  extern __shared__ unsigned long long s_tab[];                                                 \
  const bool smem_tab = a.nblk <= kSmemBlocks;                                                   \
  unsigned long long *s_base = s_tab;                                                            \
  uint32_t *s_vb = reinterpret_cast<uint32_t *>(s_tab + a.nblk);                                 \
  if (smem_tab) {                                                                                \
    for (uint32_t i = threadIdx.x; i <= a.nblk; i += blockDim.x) s_vb[i] = a.blk_vb[i];          \
    for (uint32_t i = threadIdx.x; i < a.nblk; i += blockDim.x) s_base[i] = a.blk_base[i];       \
  }                                                                                              \
  __syncthreads();                                                                               \
  const uint32_t *vb = smem_tab ? s_vb : a.blk_vb;                                               \
  const unsigned long long *bbase = smem_tab ? s_base : (const unsigned long long *)a.blk_base;

template <int ESZ>
__global__ void __launch_bounds__(256) uf_sample(MinArgs a) {
  UF_STAGE_BLOCKS();
  unsigned long long my_edges = 0, my_hbm = 0, my_link = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x) {
    uint32_t w[kUfSample], k;
    bool host;
    uf_sample_edges<ESZ>(a, vb, bbase, v, w, k, host);
    if (!k) continue;
#pragma unroll
    for (uint32_t j = 0; j < kUfSample; j++)
      if (j < k && w[j] != v) uf_union(a.val, v, w[j]);
    my_edges += k;
    if (host) my_link += (unsigned long long)k * ESZ;
    else my_hbm += (unsigned long long)k * ESZ;
  }
  my_edges = warp_sum(my_edges);
  my_hbm = warp_sum(my_hbm);
  my_link = warp_sum(my_link);
  if (lane_id() == 0 && my_edges) {
    atomicAdd(&a.ctrl->edges, my_edges);
    atomicAdd(&a.ctrl->hbm_bytes, my_hbm);
    atomicAdd(&a.ctrl->link_bytes, my_link);
  }
}

// Step 3 work items: the lists past the sample of every vertex outside the
// component of `hub` (labels are flattened roots here).
template <int ESZ>
__global__ void __launch_bounds__(256) uf_items(MinArgs a, uint32_t hub) {
  const uint32_t skip = ldcg(a.val + hub);
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nwords = (a.nv + 31) / 32;
  unsigned long long my_edges = 0, my_hbm = 0, my_link = 0;
  for (uint32_t word = gwarp; word < nwords; word += nwarps) {
    const uint32_t v = word * 32u + lane;
    uint32_t cnt = 0;
    unsigned long long eaddr = 0;
    if (v < a.nv && ldcg(a.val + v) != skip) {
      const uint64_t s = __ldg(a.off + v), e = __ldg(a.off + v + 1);
      const uint32_t deg = (uint32_t)(e - s);
      if (deg > kUfSample) {
        bool host;
        eaddr = list_addr(a.lc, __ldg(a.blk_base + find_block(a.blk_vb, a.nblk, v)), a.host_base,
                          v, s, deg, ESZ, &host);
        cnt = deg - kUfSample;
        eaddr += (unsigned long long)kUfSample * ESZ;
        my_edges += cnt;
        if (host) my_link += (unsigned long long)cnt * ESZ;
        else my_hbm += (unsigned long long)cnt * ESZ;
      }
    }
    const bool small = cnt > 0 && cnt < a.small_deg;
    const bool big = cnt >= a.small_deg;
    const unsigned sm = __ballot_sync(kFull, small);
    if (sm) {
      const int ldr = __ffs(sm) - 1;
      unsigned long long base = 0;
      if (lane == (unsigned)ldr) base = atomicAdd(&c->cnt_small[0], (unsigned long long)__popc(sm));
      base = shfl64(base, ldr);
      const unsigned long long pos = base + __popc(sm & lanemask_lt());
      if (small) {
        if (pos < a.cap_s) a.qs[pos] = make_item(eaddr, cnt, v, v);
        else atomicCAS(&c->err, 0u, kDevErrQueue);
      }
    }
    if (__any_sync(kFull, big)) {
      const unsigned nch = big ? (cnt + a.chunk - 1) / a.chunk : 0u;
      const unsigned inc = warp_incl_scan<unsigned>(nch);
      const unsigned tot = __shfl_sync(kFull, inc, 31);
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&c->cnt_big[0], (unsigned long long)tot);
      base = shfl64(base, 0);
      if (big) {
        unsigned long long pos = base + inc - nch;
        for (unsigned k = 0; k < nch; k++, pos++) {
          const uint32_t lo = k * a.chunk;
          if (pos < a.cap_b)
            a.qb[pos] = make_item(eaddr + (unsigned long long)lo * ESZ, min(a.chunk, cnt - lo), v, v);
          else
            atomicCAS(&c->err, 0u, kDevErrQueue);
        }
      }
    }
  }
  my_edges = warp_sum(my_edges);
  my_hbm = warp_sum(my_hbm);
  my_link = warp_sum(my_link);
  if (lane == 0 && my_edges) {
    atomicAdd(&c->edges, my_edges);
    atomicAdd(&c->hbm_bytes, my_hbm);
    atomicAdd(&c->link_bytes, my_link);
  }
}

template <int ESZ>
__global__ void __launch_bounds__(256) uf_unions(MinArgs a) {
  MinCtrl *c = a.ctrl;
  const unsigned lane = lane_id();
  const unsigned gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const unsigned long long ns = min(ldcg(&c->cnt_small[0]), a.cap_s);
  const unsigned long long nb = min(ldcg(&c->cnt_big[0]), a.cap_b);
  const unsigned long long ntask = nb + (ns + 31) / 32;
  constexpr int PER = 16 / ESZ;
  for (unsigned long long t = gwarp; t < ntask; t += nwarps) {
    if (t < nb) {
      // a chunk of one list: 16-byte loads, lanes outside [start, end) masked
      const MinItem it = a.qb[t];
      const uintptr_t start = it.ea_cnt & kAddrMask;
      const uintptr_t end = start + (uintptr_t)(it.ea_cnt >> 48) * ESZ;
      for (uintptr_t p = (start & ~(uintptr_t)127) + 16u * lane; p < end; p += 512u) {
        const uint4 q = ld_nc_v4(p);
        const uint32_t f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < PER; j++) {
          const uintptr_t ea = p + (uintptr_t)ESZ * j;
          if (ea >= start && ea < end)
            uf_union(a.val, it.v, ESZ == 4 ? edge_dst(f[j], a.wshift) : f[2 * j]);
        }
      }
    } else {
      // 32 short suffixes, their edges spread over the lanes
      const unsigned long long idx = (t - nb) * 32ull + lane;
      MinItem it{0, 0, 0};
      if (idx < ns) it = a.qs[idx];
      const unsigned cnt = (unsigned)(it.ea_cnt >> 48);
      const unsigned long long eaddr = it.ea_cnt & kAddrMask;
      const unsigned incl = warp_incl_scan<unsigned>(cnt);
      const unsigned excl = incl - cnt;
      const unsigned total = __shfl_sync(kFull, incl, 31);
      for (unsigned k = 0; k < total; k += 32) {
        const unsigned tt = k + lane;
        const int o = warp_owner(excl, tt);
        const unsigned long long ea = shfl64(eaddr, o);
        const unsigned oex = __shfl_sync(kFull, excl, o);
        const uint32_t ou = __shfl_sync(kFull, it.v, o);
        if (tt < total) {
          const uint32_t raw = ld_nc_u32((uintptr_t)ea + (uintptr_t)(tt - oex) * ESZ);
          uf_union(a.val, ou, ESZ == 4 ? edge_dst(raw, a.wshift) : raw);
        }
      }
    }
  }
}

__global__ void uf_flatten(uint32_t *p, uint32_t nv) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    uint32_t r = ldcg(p + v);
    while (true) {
      const uint32_t n = ldcg(p + r);
      if (n == r) break;
      r = n;
    }
    p[v] = r;
  }
}

__global__ void uf_init(MinArgs a) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += gridDim.x * blockDim.x)
    a.val[v] = v;
  if (blockIdx.x == 0 && threadIdx.x == 0) memset(a.ctrl, 0, sizeof(MinCtrl));
}

// ------------------------------------------------------------------ host --

// Chunk items one phase can queue.  Each vertex is queued at most once per
// phase, and a vertex of degree >= small, or (queue mode) whose list is
// read over the host link -- a host block, degree >= the small-list cache's
// bound -- yields ceil(deg / chunk) items: at most ne / chunk plus the
// number of such vertices, which is at most ne / small plus the host
// edges / the cache bound (and at most nv).
static uint64_t chunk_capacity(const thv_graph *g, uint32_t chunk, uint32_t small) {
  const uint64_t host_edges = g->plan.host_edge_bytes / std::max<uint32_t>(g->esz, 1);
  const uint64_t host_lists =
      std::min<uint64_t>(g->nv, host_edges / std::max<uint32_t>(g->plan.list_deg, 1));
  return g->ne / chunk + g->ne / std::max<uint32_t>(small, 1) + host_lists + 64;
}

static thv_status ensure_min_state(thv_graph *g, uint32_t chunk,
                                   uint32_t small) {
  MinState *&ms = g->ms;
  // reuse the state while its chunk queue holds this configuration's items
  // (BFS/CC and SSSP default to different chunk sizes on one graph)
  const uint64_t need_b = chunk_capacity(g, chunk, small);
  if (ms && ms->valid && ms->nv == g->nv && ms->cap_b >= need_b) return THV_OK;
  if (ms) minprop_free(g);
  ms = new MinState();
  ms->nv = g->nv;
  ms->chunk = chunk;
  ms->small = small;
  const uint64_t nw = (g->nv + 31) / 32;
  ms->ngroups = (uint32_t)((nw + 31) / 32);
  const uint64_t nw_alloc = (uint64_t)ms->ngroups * 32;
  ms->cap_s = g->nv + 32;
  ms->cap_b = need_b;
  THV_TRY(dev_alloc((void **)&ms->d_val, g->nv * 4 + 64, "values"));
  THV_TRY(dev_alloc((void **)&ms->d_bm, nw_alloc * 4, "pending bitmap"));
  THV_TRY(dev_alloc((void **)&ms->d_wmin, nw_alloc * 4, "pending minima"));
  THV_TRY(dev_alloc((void **)&ms->d_bm2, nw_alloc * 4, "frontier copy"));
  THV_TRY(dev_alloc((void **)&ms->d_flist, 3 * kLocalCap * 4, "small-frontier lists"));
  THV_TRY(dev_alloc((void **)&ms->d_qs, ms->cap_s * sizeof(MinItem), "queue"));
  THV_TRY(dev_alloc((void **)&ms->d_qb, ms->cap_b * sizeof(MinItem), "chunk queue"));
  THV_TRY(dev_alloc((void **)&ms->d_qs2, ms->cap_s * sizeof(MinItem), "queue"));
  THV_TRY(dev_alloc((void **)&ms->d_qb2, ms->cap_b * sizeof(MinItem), "chunk queue"));
  THV_TRY(dev_alloc((void **)&ms->d_qbits, nw_alloc * 2 * 4, "queued-vertex bitmaps"));
  THV_TRY(dev_alloc((void **)&ms->d_ctrl, sizeof(MinCtrl), "control"));
  THV_TRY(pinned_alloc((void **)&ms->h_ctrl, sizeof(MinCtrl), "control"));
  THV_CUDA(cudaEventCreate(&ms->ev0));
  THV_CUDA(cudaEventCreate(&ms->ev1));
  ms->valid = true;
  return THV_OK;
}

void minprop_free(thv_graph *g) {
  MinState *ms = g->ms;
  if (!ms) return;
  dev_free(ms->d_val);
  dev_free(ms->d_bm);
  dev_free(ms->d_wmin);
  dev_free(ms->d_bm2);
  dev_free(ms->d_flist);
  dev_free(ms->d_qs);
  dev_free(ms->d_qb);
  dev_free(ms->d_qs2);
  dev_free(ms->d_qb2);
  dev_free(ms->d_qbits);
  dev_free(ms->d_ctrl);
  pinned_free(ms->h_ctrl);
  if (ms->ev0) cudaEventDestroy(ms->ev0);
  if (ms->ev1) cudaEventDestroy(ms->ev1);
  delete ms;
  g->ms = nullptr;
}

template <int OP, int ESZ>
static thv_status launch_minprop(thv_graph *g, MinArgs &a, cudaStream_t st,
                                 uint32_t &launches, bool scan_mode) {
  auto kern = scan_mode ? (OP == OP_BFS && a.do_alpha ? bfs_do_kernel<ESZ> : minprop_kernel<OP, ESZ>)
                        : minq_kernel<OP, ESZ>;
  const size_t nb = g->plan.blocks.size();
  const size_t smem = nb <= kSmemBlocks ? nb * 8 + (nb + 1) * 4 : 0;
  THV_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int bpsm = 0;
  THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern,
                                                         kMinThreads, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "minprop kernel cannot be resident");
  const int grid = bpsm * g->num_sms;
  const uint32_t nw_alloc = g->ms->ngroups * 32u;
  const int init_grid = std::max(1, std::min<int>(g->num_sms * 8,
                                (int)((g->nv + 255) / 256)));
  minprop_init<OP><<<init_grid, 256, 0, st>>>(a, nw_alloc);
  if (!scan_mode && OP != OP_BFS) {
    minq_clear<<<init_grid, 256, 0, st>>>(a.qbits, a.ngroups * 64u);
    launches++;
  }
  THV_CUDA(cudaGetLastError());
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel((void *)kern, dim3(grid),
                                       dim3(kMinThreads), args, smem, st));
  launches += 2;
  return THV_OK;
}

thv_status run_minprop(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                       cudaStream_t st, thv_stats *stats) {
  const int op = algo == THV_ALGO_BFS ? OP_BFS : algo == THV_ALGO_CC ? OP_CC : OP_SSSP;
  if (op == OP_SSSP && !g->weighted)
    return fail(THV_EINVAL, "SSSP needs edge weights (WCSR, or CSR opened "
                            "with THV_OPEN_WEIGHTS)");
  if (g->fmt == THV_FMT_CSC)
    return fail(THV_EINVAL, "BFS/CC/SSSP need out-edges (CSR/WCSR), got CSC");
  if (g->nv >= 0xFFFFFFFFull)
    return fail(THV_EUNSUPPORTED, "vertex count %llu exceeds u32 values",
                (unsigned long long)g->nv);
  const uint32_t src = o ? o->source : 1;
  if (op != OP_CC && src >= g->nv)
    return fail(THV_EINVAL, "source %u out of range (n=%llu)", src,
                (unsigned long long)g->nv);
  // edges per chunk item by mode: queue mode (SSSP by default) 2 KiB --
  // RMAT-24 SSSP on packed 4-byte edges: 512 edges 7.34 ms, 256 7.66 ms --
  // and scan mode 4 KiB
  bool queue_mode = op == OP_SSSP;
  if (o && (o->flags & THV_RUN_SCAN_COMPACTION)) queue_mode = false;
  if (o && (o->flags & THV_RUN_QUEUE_COMPACTION)) queue_mode = true;
  uint32_t chunk = o && o->chunk_edges
                       ? o->chunk_edges
                       : (queue_mode ? kQueueChunkBytes : kScanChunkBytes) / g->esz;
  chunk = std::min<uint32_t>(32768, std::max<uint32_t>(32, (chunk + 31) / 32 * 32));
  const uint32_t small = std::min<uint32_t>(
      32768, o && o->small_degree ? o->small_degree : (queue_mode ? kQueueSmall : kDefaultSmall));
  THV_TRY(ensure_plan(g));
  // work items keep edge addresses in 48 bits
  const uint64_t top = std::max<uint64_t>(g->h_edges_dev + g->h_edges_bytes,
                                          (uint64_t)g->plan.d_resident + g->plan.d_resident_bytes);
  if (top >> 48) return fail(THV_EUNSUPPORTED, "edge address above 2^48");
  THV_TRY(ensure_min_state(g, chunk, small));
  MinState *ms = g->ms;

  MinArgs a{};
  a.val = ms->d_val;
  a.bm = ms->d_bm;
  a.wmin = ms->d_wmin;
  a.off = g->d_off;
  a.blk_vb = g->plan.d_vbegin;
  a.blk_base = g->plan.d_base;
  a.host_base = g->h_edges_dev;
  a.host_end = g->h_edges_dev + g->h_edges_bytes;
  a.lc = list_cache_of(g->plan);
  a.blk_access = g->plan.d_access;
  a.qs = ms->d_qs;
  a.qb = ms->d_qb;
  a.qs2 = ms->d_qs2;
  a.qb2 = ms->d_qb2;
  a.qbits = ms->d_qbits;
  a.cap_s = ms->cap_s;
  a.cap_b = ms->cap_b;
  a.ctrl = ms->d_ctrl;
  const uint32_t tmo = o && o->timeout_ms ? o->timeout_ms : 60000u;
  a.timeout_ns = (unsigned long long)tmo * 1000000ull;
  a.nblk = (uint32_t)g->plan.blocks.size();
  a.nv = (uint32_t)g->nv;
  a.ngroups = ms->ngroups;
  a.max_iters = (uint32_t)std::min<uint64_t>(g->nv + 2, 0xFFFFFFF0ull) * 2 + 8;
  a.delta = o && o->sssp_delta ? o->sssp_delta : (op == OP_CC ? 1u : kDefaultDelta);
  a.growth = op == OP_CC ? kCcGrowth : (o && o->sssp_growth ? o->sssp_growth : kSsspGrowth);
  a.wshift = g->wshift;
  a.wbase = g->wbase;
  a.small_deg = small;
  a.chunk = chunk;
  a.src = src;
  a.ne = g->ne;
  a.link_every = kLinkEvery;

  // scan-built queues keep vertex order (coalesced offset reads) and no
  // fences: better for BFS and CC; SSSP gains from fewer barriers
  bool scan_mode = op != OP_SSSP;
  if (o && (o->flags & THV_RUN_SCAN_COMPACTION)) scan_mode = true;
  if (o && (o->flags & THV_RUN_QUEUE_COMPACTION)) scan_mode = false;
  // Direction-optimising BFS when every out-edge is resident: bottom-up
  // levels scan an in-edge transpose held in HBM (built once per graph,
  // outside the timed region)
  if (op == OP_BFS && scan_mode && !(o && (o->flags & THV_RUN_TOP_DOWN_ONLY)) &&
      g->plan.host_edge_bytes == 0 && g->ne > 0) {
    THV_TRY(ensure_transpose(g, st));
    a.in_off = g->d_in_off;
    a.in_adj = g->d_in_adj;
    a.bm2 = ms->d_bm2;
    a.flist = ms->d_flist;
    a.do_alpha = kBfsAlpha;
    a.do_beta = kBfsBeta;
  }

  uint32_t launches = 0;
  THV_CUDA(cudaEventRecord(ms->ev0, st));
  thv_status s = THV_OK;
  // CC of a symmetric graph: sampling union-find (same labels as min-label
  // propagation, most lists never read)
  const bool union_find = op == OP_CC && g->symmetric && g->nv > 0 &&
                          !(o && (o->flags & THV_RUN_LABEL_PROPAGATION));
  if (union_find) {
    const int grid = g->num_sms * 8;
    const uint32_t hub = g->hub_vertex();
    const size_t nb = g->plan.blocks.size();
    const size_t smem = nb <= kSmemBlocks ? nb * 8 + (nb + 1) * 4 : 0;
    uf_init<<<grid, 256, 0, st>>>(a);
    if (g->esz == 4) uf_sample<4><<<grid, 256, smem, st>>>(a);
    else uf_sample<8><<<grid, 256, smem, st>>>(a);
    uf_flatten<<<grid, 256, 0, st>>>(a.val, a.nv);
    if (g->esz == 4) {
      uf_items<4><<<grid, 256, 0, st>>>(a, hub);
      uf_unions<4><<<grid, 256, 0, st>>>(a);
    } else {
      uf_items<8><<<grid, 256, 0, st>>>(a, hub);
      uf_unions<8><<<grid, 256, 0, st>>>(a);
    }
    uf_flatten<<<grid, 256, 0, st>>>(a.val, a.nv);
    THV_CUDA(cudaGetLastError());
    launches += 6;
  } else if (g->esz == 4) {
    if (op == OP_BFS) s = launch_minprop<OP_BFS, 4>(g, a, st, launches, scan_mode);
    else if (op == OP_CC) s = launch_minprop<OP_CC, 4>(g, a, st, launches, scan_mode);
    else s = launch_minprop<OP_SSSP, 4>(g, a, st, launches, scan_mode);  // packed weights
  } else {
    if (op == OP_BFS) s = launch_minprop<OP_BFS, 8>(g, a, st, launches, scan_mode);
    else if (op == OP_CC) s = launch_minprop<OP_CC, 8>(g, a, st, launches, scan_mode);
    else s = launch_minprop<OP_SSSP, 8>(g, a, st, launches, scan_mode);
  }
  if (s != THV_OK) return s;
  THV_CUDA(cudaEventRecord(ms->ev1, st));
  const bool want_sum = o && (o->flags & THV_RUN_CHECKSUM);
  if (want_sum) {
    const int cgrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
    values_checksum_kernel<<<cgrid, 256, 0, st>>>(ms->d_val, g->nv, &ms->d_ctrl->checksum);
    THV_CUDA(cudaGetLastError());
    launches++;
  }
  THV_CUDA(cudaMemcpyAsync(ms->h_ctrl, ms->d_ctrl, sizeof(MinCtrl),
                           cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaStreamSynchronize(st));
  const MinCtrl &hc = *ms->h_ctrl;
  g->last_algo = algo;
  if (stats) {
    float ms_ = 0.f;
    cudaEventElapsedTime(&ms_, ms->ev0, ms->ev1);
    stats->device_ms = ms_;
    stats->iterations = hc.iters;
    stats->edges_expanded = hc.edges;
    stats->hbm_edge_bytes = hc.hbm_bytes;
    stats->link_edge_bytes = hc.link_bytes;
    stats->kernel_launches = launches;
    stats->d2h_bytes += sizeof(MinCtrl);
    stats->checksum = want_sum ? hc.checksum : 0;
    stats->bottom_up_levels = hc.bu_levels;
  }
  if (hc.err == kDevErrBarrier)
    return fail(THV_ETIMEOUT, "grid barrier wait exceeded %u ms", tmo);
  if (hc.err == kDevErrIters)
    return fail(THV_ETIMEOUT, "iteration cap %u reached", a.max_iters);
  if (hc.err == kDevErrQueue)
    return fail(THV_EDEVICE, "work queue overflow");
  if (hc.err) return fail(THV_EDEVICE, "device error %u", hc.err);
  return THV_OK;
}

thv_status minprop_values(thv_graph *g, uint32_t *out, cudaStream_t st) {
  if (!g->ms || !g->ms->valid) return fail(THV_EINVAL, "no values: nothing ran");
  THV_CUDA(cudaMemcpyAsync(out, g->ms->d_val, g->nv * 4, cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaStreamSynchronize(st));
  return THV_OK;
}

const uint32_t *minprop_device_values(thv_graph *g) {
  return g->ms ? g->ms->d_val : nullptr;
}

}  // namespace thv

// ============================================== allocation-free BFS entry
//
// thv_bfs_noalloc runs the same BFS kernel as thv_run over a CSR that the
// caller already holds in device (or host-mapped) memory, writing into the
// caller's value array, and allocates nothing: its scratch (control block,
// one-entry block table, pending bitmap, work queues) lives in the
// file-scope array below, which every GPU that loads this library holds
// until the process exits.  It exists for callers that cannot call
// cudaMalloc on this path: a host framework that owns all device memory
// through its own pool or arena, or a latency-critical path that cannot
// afford cudaMalloc/cudaFree's implicit device synchronisation.
//
// All calls share the one array: the kernel reinitialises what must start
// at zero (bitmap, counters) on every call, and calls whose work overlaps
// on the GPU (concurrent streams, or several host threads) race on it --
// serialise them.  The first call on a device looks up the array's device
// address (cudaGetSymbolAddress) and the device's SM count; make that first
// call before any stream capture.  The address is kept for the life of the
// process, so a cudaDeviceReset after the first call is not supported.
namespace thv {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code may not take the array's address directly (a host-side shadow,
// not a device address): this is the looked-up device address per device,
// with that device's SM count.
static std::mutex g_noalloc_mu;
static uintptr_t g_noalloc_addr[64];
static int g_noalloc_sms[64];

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct NoAllocLayout {
  size_t ctrl, table_vb, table_base, bm, qs, qb, total;
  uint32_t ngroups;
  uint64_t cap_s, cap_b;
};

static NoAllocLayout noalloc_layout(uint64_t nv, uint64_t ne) {
  NoAllocLayout l{};
  const uint64_t nw = (nv + 31) / 32;
  l.ngroups = (uint32_t)((nw + 31) / 32);
  l.cap_s = nv + 32;
  l.cap_b = ne / kDefaultChunk + ne / kDefaultSmall + 64;
  size_t off = 0;
  l.ctrl = off;       off += align256(sizeof(MinCtrl));
  l.table_vb = off;   off += align256(2 * sizeof(uint32_t));
  l.table_base = off; off += align256(sizeof(uint64_t));
  l.bm = off;         off += align256((size_t)l.ngroups * 32 * 4);
  l.qs = off;         off += align256(l.cap_s * sizeof(MinItem));
  l.qb = off;         off += align256(l.cap_b * sizeof(MinItem));
  l.total = off;
  return l;
}

// One edge block covering the whole graph, at the caller's adjacency.
__global__ void noalloc_table_init(uint32_t *vb, uint64_t *base, uint32_t nv, uint64_t adj) {
  vb[0] = 0;
  vb[1] = nv;
  base[0] = adj;
}

static thv_status noalloc_scratch_address(int dev, uintptr_t *addr, int *sms) {
  if (dev < 0 || dev >= 64) return fail(THV_EUNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(THV_ECUDA, "cudaGetSymbolAddress(no-alloc scratch): %s", cudaGetErrorString(e));
    int n = 0;
    THV_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    g_noalloc_sms[dev] = n;
    g_noalloc_addr[dev] = (uintptr_t)p;
  }
  *addr = g_noalloc_addr[dev];
  *sms = g_noalloc_sms[dev];
  return THV_OK;
}

static thv_status bfs_noalloc(const uint64_t *d_off, const uint32_t *d_adj, uint64_t nv,
                              uint64_t ne, uint32_t source, uint32_t *d_values,
                              cudaStream_t st, uint64_t *iterations) {
  if (!d_off || (!d_adj && ne) || !d_values) return fail(THV_EINVAL, "null argument");
  if (nv == 0 || nv >= 0xFFFFFFFFull) return fail(THV_EINVAL, "vertex count %llu out of range",
                                                  (unsigned long long)nv);
  if (source >= nv) return fail(THV_EINVAL, "source %u out of range (n=%llu)", source,
                                (unsigned long long)nv);
  if ((uintptr_t)d_adj % 128 != 0)
    return fail(THV_EINVAL, "adjacency array must be 128-byte aligned");
  if (((uintptr_t)d_adj + ne * 4) >> 48) return fail(THV_EUNSUPPORTED, "edge address above 2^48");
  const NoAllocLayout l = noalloc_layout(nv, ne);
  if (l.total > kNoAllocScratchBytes)
    return fail(THV_ENOMEM, "graph (n=%llu, m=%llu) needs %zu bytes of scratch; the "
                "allocation-free entry point holds %zu", (unsigned long long)nv,
                (unsigned long long)ne, l.total, kNoAllocScratchBytes);
  int dev = 0;
  THV_CUDA(cudaGetDevice(&dev));
  uintptr_t base = 0;
  int sms = 0;
  THV_TRY(noalloc_scratch_address(dev, &base, &sms));

  MinArgs a{};
  a.val = d_values;
  a.bm = (uint32_t *)(base + l.bm);
  a.wmin = nullptr;  // BFS keeps no pending minima
  a.off = d_off;
  a.blk_vb = (const uint32_t *)(base + l.table_vb);
  a.blk_base = (const uint64_t *)(base + l.table_base);
  a.host_base = 0;
  a.host_end = 0;
  a.qs = (MinItem *)(base + l.qs);
  a.qb = (MinItem *)(base + l.qb);
  a.cap_s = l.cap_s;
  a.cap_b = l.cap_b;
  a.ctrl = (MinCtrl *)(base + l.ctrl);
  a.timeout_ns = 60000ull * 1000000ull;
  a.nblk = 1;
  a.nv = (uint32_t)nv;
  a.ngroups = l.ngroups;
  a.max_iters = (uint32_t)std::min<uint64_t>(nv + 2, 0xFFFFFFF0ull) * 2 + 8;
  a.delta = 1;
  a.small_deg = kDefaultSmall;
  a.chunk = kDefaultChunk;
  a.src = source;
  a.growth = kCcGrowth;

  noalloc_table_init<<<1, 1, 0, st>>>((uint32_t *)a.blk_vb, (uint64_t *)a.blk_base, (uint32_t)nv,
                                      (uint64_t)(uintptr_t)d_adj);
  const int init_grid = std::max(1, std::min<int>(sms * 8, (int)((nv + 255) / 256)));
  minprop_init<OP_BFS><<<init_grid, 256, 0, st>>>(a, l.ngroups * 32u);
  THV_CUDA(cudaGetLastError());
  auto kern = minprop_kernel<OP_BFS, 4>;
  const size_t smem = 1 * 8 + 2 * 4;
  // thv_run sets this kernel's dynamic shared memory limit per plan (down
  // to 0 for large block tables); this launch needs its own
  THV_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  int bpsm = 0;
  THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, kMinThreads, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "BFS kernel cannot be resident");
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel((void *)kern, dim3(bpsm * sms),
                                       dim3(kMinThreads), args, smem, st));
  MinCtrl hc;  // the caller's stack: nothing allocated
  THV_CUDA(cudaMemcpyAsync(&hc, a.ctrl, sizeof(MinCtrl), cudaMemcpyDeviceToHost, st));
  THV_CUDA(cudaStreamSynchronize(st));
  if (iterations) *iterations = hc.iters;
  if (hc.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "grid barrier wait timed out");
  if (hc.err == kDevErrIters) return fail(THV_ETIMEOUT, "iteration cap reached");
  if (hc.err == kDevErrQueue) return fail(THV_EDEVICE, "work queue overflow");
  if (hc.err) return fail(THV_EDEVICE, "device error %u", hc.err);
  return THV_OK;
}

}  // namespace thv

extern "C" thv_status thv_bfs_noalloc(const uint64_t *d_off, const uint32_t *d_adj, uint64_t nv,
                                      uint64_t ne, uint32_t source, uint32_t *d_values,
                                      void *stream, uint64_t *iterations) {
  try {
    return thv::bfs_noalloc(d_off, d_adj, nv, ne, source, d_values, (cudaStream_t)stream,
                            iterations);
  } catch (...) {
    return thv::fail(THV_EINVAL, "exception in thv_bfs_noalloc");
  }
}
