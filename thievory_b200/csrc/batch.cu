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
//   SSSP dist[w][s] rows of 64 u32 (vertex-major, one 256-byte row per
//        vertex); per edge and source in the mask the single-source
//        relaxation "cand < dist => atomicMin, mark pending" with the same
//        near/far window, shared by all sources.
// Results are bit-identical to single-source runs: BFS levels are exact
// (level-synchronous), SSSP is the unique min fixed point.
#include <algorithm>
#include <cstring>
#include <vector>

#include "thv_device.cuh"
#include "thv_internal.h"

namespace thv {

enum { MS_BFS = 0, MS_SSSP = 1 };
constexpr int kMsThreads = 512;
constexpr uint32_t kMsWidth = 64;       // sources per group (mask bits)
constexpr uint32_t kMaxBfsLevel = 254;  // u8 level bytes hold level + 1

struct MsCtrl {
  GridBar bar;
  unsigned err, iters;
  unsigned long long cnt_small[3], cnt_big[3], remaining[3], wc[3];
  unsigned minkept[3], pad;
  unsigned long long edges, hbm_bytes, link_bytes, pairs;
};

struct MsArgs {
  const uint64_t *off;
  const uint32_t *blk_vb;
  const uint64_t *blk_base;
  uint64_t host_base;
  unsigned long long *visit;  // BFS
  unsigned long long *front;  // pending (vertex, source) pairs
  uint8_t *lvl;               // BFS [nv][64]: level + 1, 0 = unreached
  uint32_t *dist;             // SSSP [nv][64]: distance + 1
  uint32_t *bm;
  uint32_t *wmin;             // SSSP: lower bound of pending distances per word
  WorkItem *qs, *qb;
  unsigned long long *qsm, *qbm;  // masks of the queued items
  unsigned long long cap_s, cap_b;
  MsCtrl *ctrl;
  const uint32_t *sources;
  unsigned long long timeout_ns;
  uint32_t nblk, nv, ngroups, max_iters;
  uint32_t small_deg, chunk, delta, k;
};

struct BatchState {
  uint64_t nv = 0;
  uint32_t chunk = 0, small = 0;
  bool sssp = false;
  unsigned long long *d_visit = nullptr, *d_front = nullptr;
  uint8_t *d_lvl = nullptr;
  uint32_t *d_dist = nullptr;
  uint32_t *d_bm = nullptr, *d_wmin = nullptr;
  WorkItem *d_qs = nullptr, *d_qb = nullptr;
  unsigned long long *d_qsm = nullptr, *d_qbm = nullptr;
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

// SSSP edge u->w of weight wt for the sources in f.
__device__ __forceinline__ void ms_sssp_edge(const MsArgs &a, uint32_t u, uint32_t w,
                                             uint32_t wt, unsigned long long f) {
  const uint32_t *du = a.dist + (size_t)u * kMsWidth;
  uint32_t *dw = a.dist + (size_t)w * kMsWidth;
  unsigned long long improved = 0;
  uint32_t best = 0xFFFFFFFFu;
  while (f) {
    const int s = __ffsll((long long)f) - 1;
    f &= f - 1;
    const unsigned long long cand = (unsigned long long)ldcg(du + s) + wt;
    if (cand < ldcg(dw + s)) {
      const uint32_t old = atomicMin(dw + s, (uint32_t)cand);
      if (cand < old) {
        improved |= 1ull << s;
        best = min(best, (uint32_t)cand);
      }
    }
  }
  if (improved) {
    atomicOr(a.front + w, improved);
    atomicMin(a.wmin + (w >> 5), best);
    mark_pending<MS_SSSP>(a, w);
  }
}

template <int OP, int ESZ>
__device__ __forceinline__ void ms_edge(const MsArgs &a, uint32_t u, uint32_t w,
                                        uint32_t wt, unsigned long long f, uint32_t lvl1) {
  if (OP == MS_BFS) ms_bfs_edge(a, w, f, lvl1);
  else ms_sssp_edge(a, u, w, wt, f);
}

template <int OP, int ESZ>
__device__ __forceinline__ void ms_chunk(const MsArgs &a, const WorkItem &it,
                                         unsigned long long f, uint32_t lvl1) {
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
        ms_edge<OP, ESZ>(a, it.v, ESZ == 4 ? e[j] : e[2 * j], ESZ == 4 ? 1u : e[2 * j + 1], f, lvl1);
    }
  }
}

template <int OP, int ESZ>
__device__ __forceinline__ void ms_group(const MsArgs &a, unsigned long long first,
                                         unsigned long long n_small, uint32_t lvl1) {
  const unsigned lane = lane_id();
  const unsigned long long idx = first + lane;
  WorkItem it{0, 0, 0};
  unsigned long long f = 0;
  if (idx < n_small) {
    it = a.qs[idx];
    f = a.qsm[idx];
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
        ms_edge<OP, ESZ>(a, ou, ld_nc_u32(addr), 1u, of, lvl1);
      } else {
        const uint2 e = ld_nc_u2(addr);
        ms_edge<OP, ESZ>(a, ou, e.x, e.y, of, lvl1);
      }
    }
  }
}

template <int OP, int ESZ>
__global__ void __launch_bounds__(kMsThreads) ms_kernel(MsArgs a) {
  extern __shared__ uint32_t s_vb[];
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
  unsigned iter = 0, level = 1;  // BFS level of the vertices being expanded
  for (;; ++iter) {
    if (iter >= a.max_iters || (OP == MS_BFS && level > kMaxBfsLevel)) {
      if (leader) atomicCAS(&c->err, 0u, OP == MS_BFS && level > kMaxBfsLevel ? kDevErrDepth : kDevErrIters);
      break;
    }
    const unsigned slot = iter % 3, nslot = (iter + 1) % 3;
    if (leader) {
      c->cnt_small[nslot] = 0;
      c->cnt_big[nslot] = 0;
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
            const uint32_t *dv = a.dist + (size_t)v * kMsWidth;
            unsigned long long r = f;
            while (r) {
              const int s = __ffsll((long long)r) - 1;
              r &= r - 1;
              const uint32_t d = ldcg(dv + s);
              if (d < thr) take |= 1ull << s;
              else kmin = min(kmin, d);
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
          const uint32_t b = find_block(vb, a.nblk, v);
          const unsigned long long base = __ldg(a.blk_base + b);
          eaddr = base + s0 * ESZ;
          my_edges += deg;
          my_pairs += __popcll(take);
          if (base == a.host_base) my_link += (unsigned long long)deg * ESZ;
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
    if (ns + nb == 0) {
      if (OP == MS_BFS) break;
      if (ldcg(&c->remaining[slot]) == 0) break;
      thr = (uint32_t)min((unsigned long long)ldcg(&c->minkept[slot]) + a.delta, 0xFFFFFFFFull);
      continue;
    }
    // ----------------------------------------------------------- expansion
    const uint32_t lvl1 = level + 1;
    const unsigned long long ntask = nb + (ns + 31) / 32;
    for (unsigned long long t = gwarp; t < ntask;) {
      if (t < nb) ms_chunk<OP, ESZ>(a, a.qb[t], a.qbm[t], lvl1);
      else ms_group<OP, ESZ>(a, (t - nb) * 32ull, ns, lvl1);
      unsigned long long nt = 0;
      if (lane == 0) nt = nwarps + atomicAdd(&c->wc[slot], 1ull);
      t = shfl64(nt, 0);
    }
    level++;
    if (!grid_sync(&c->bar, &c->err, a.timeout_ns)) break;
  }
  if (leader) c->iters = iter;
}

template <int OP>
__global__ void ms_init(MsArgs a, uint32_t nw_alloc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t v = tid; v < a.nv; v += stride) {
    a.front[v] = 0;
    if (OP == MS_BFS) {
      a.visit[v] = 0;
      reinterpret_cast<uint4 *>(a.lvl + v * kMsWidth)[0] = make_uint4(0, 0, 0, 0);
      reinterpret_cast<uint4 *>(a.lvl + v * kMsWidth)[1] = make_uint4(0, 0, 0, 0);
      reinterpret_cast<uint4 *>(a.lvl + v * kMsWidth)[2] = make_uint4(0, 0, 0, 0);
      reinterpret_cast<uint4 *>(a.lvl + v * kMsWidth)[3] = make_uint4(0, 0, 0, 0);
    } else {
      uint4 *row = reinterpret_cast<uint4 *>(a.dist + v * kMsWidth);
      const uint32_t inf = a.nv + 1u;
      for (int i = 0; i < 16; i++) row[i] = make_uint4(inf, inf, inf, inf);
    }
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
  if (s >= a.k) return;
  const uint32_t v = a.sources[s];
  atomicOr(a.front + v, 1ull << s);
  atomicOr(a.bm + (v >> 5), 1u << (v & 31u));
  if (OP == MS_BFS) {
    atomicOr(a.visit + v, 1ull << s);
    a.lvl[(size_t)v * kMsWidth + s] = 1;
  } else {
    a.dist[(size_t)v * kMsWidth + s] = 1;
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

// Per-source values in the single-source encoding: optional k x nv output
// (rows per source) and a checksum per source (sum of value_hash(v, val)).
template <int OP>
__global__ void ms_extract(MsArgs a, uint32_t *out, unsigned long long *sums) {
  __shared__ unsigned long long s_sum[kMsWidth];
  __shared__ uint32_t tile[32][kMsWidth + 1];
  for (uint32_t i = threadIdx.x; i < kMsWidth; i += blockDim.x) s_sum[i] = 0;
  __syncthreads();
  const uint32_t inf = a.nv + 1u;
  // blockDim = 256: 32 vertices x 64 sources per tile
  for (uint64_t base = (uint64_t)blockIdx.x * 32; base < a.nv; base += (uint64_t)gridDim.x * 32) {
    for (uint32_t i = threadIdx.x; i < 32 * kMsWidth; i += blockDim.x) {
      const uint32_t dv = i / kMsWidth, s = i % kMsWidth;
      const uint64_t v = base + dv;
      uint32_t val = inf;
      if (v < a.nv) {
        if (OP == MS_BFS) {
          const uint8_t l = a.lvl[v * kMsWidth + s];
          val = l ? l : inf;
        } else {
          val = a.dist[v * kMsWidth + s];
        }
      }
      tile[dv][s] = val;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 32 * kMsWidth; i += blockDim.x) {
      const uint32_t s = i / 32, dv = i % 32;
      const uint64_t v = base + dv;
      if (s < a.k && v < a.nv) {
        const uint32_t val = tile[dv][s];
        if (out) out[(uint64_t)s * a.nv + v] = val;
        if (sums) atomicAdd(&s_sum[s], value_hash((uint32_t)v, val));
      }
    }
    __syncthreads();
  }
  if (sums)
    for (uint32_t i = threadIdx.x; i < a.k; i += blockDim.x)
      if (s_sum[i]) atomicAdd(sums + i, s_sum[i]);
}

// ------------------------------------------------------------------ host --

void batch_free(thv_graph *g) {
  BatchState *b = g->bs;
  if (!b) return;
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
  g->bs = nullptr;
}

static thv_status ensure_batch_state(thv_graph *g, bool sssp, uint32_t chunk,
                                     uint32_t small, bool want_out) {
  BatchState *&b = g->bs;
  if (b && b->sssp == sssp && b->chunk == chunk && b->small == small &&
      (!want_out || b->d_out))
    return THV_OK;
  batch_free(g);
  b = new BatchState();
  b->nv = g->nv;
  b->sssp = sssp;
  b->chunk = chunk;
  b->small = small;
  const uint64_t nw = (g->nv + 31) / 32;
  b->ngroups = (uint32_t)((nw + 31) / 32);
  const uint64_t nw_alloc = (uint64_t)b->ngroups * 32;
  b->cap_s = g->nv + 32;
  b->cap_b = g->ne / chunk + g->ne / std::max<uint32_t>(small, 1) + 64;
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
  THV_TRY(dev_alloc((void **)&b->d_qb, b->cap_b * sizeof(WorkItem), "batch chunk queue"));
  THV_TRY(dev_alloc((void **)&b->d_qbm, b->cap_b * 8, "batch chunk masks"));
  THV_TRY(dev_alloc((void **)&b->d_ctrl, sizeof(MsCtrl), "batch control"));
  THV_TRY(pinned_alloc((void **)&b->h_ctrl, sizeof(MsCtrl), "batch control"));
  THV_TRY(dev_alloc((void **)&b->d_sources, kMsWidth * 4, "batch sources"));
  THV_TRY(pinned_alloc((void **)&b->h_sources, kMsWidth * 4, "batch sources"));
  THV_TRY(dev_alloc((void **)&b->d_sums, kMsWidth * 8, "batch checksums"));
  THV_TRY(pinned_alloc((void **)&b->h_sums, kMsWidth * 8, "batch checksums"));
  if (want_out) THV_TRY(dev_alloc((void **)&b->d_out, (uint64_t)kMsWidth * g->nv * 4 + 64, "batch output"));
  THV_CUDA(cudaEventCreate(&b->ev0));
  THV_CUDA(cudaEventCreate(&b->ev1));
  return THV_OK;
}

template <int OP, int ESZ>
static thv_status launch_group(thv_graph *g, MsArgs &a, cudaStream_t st, bool want_out,
                               uint32_t &launches) {
  BatchState *b = g->bs;
  auto kern = ms_kernel<OP, ESZ>;
  const size_t smem = g->plan.vbegin.size() <= kSmemBlocks + 1 ? g->plan.vbegin.size() * 4 : 0;
  int bpsm = 0;
  THV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, kMsThreads, smem));
  if (bpsm < 1) return fail(THV_ECUDA, "batch kernel cannot be resident");
  const int grid = bpsm * g->num_sms;
  const int igrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 255) / 256)));
  THV_CUDA(cudaMemcpyAsync(b->d_sources, b->h_sources, kMsWidth * 4, cudaMemcpyHostToDevice, st));
  ms_init<OP><<<igrid, 256, 0, st>>>(a, b->ngroups * 32u);
  ms_seed<OP><<<1, kMsWidth, 0, st>>>(a);
  THV_CUDA(cudaGetLastError());
  void *args[] = {&a};
  THV_CUDA(cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(kMsThreads), args, smem, st));
  THV_CUDA(cudaMemsetAsync(b->d_sums, 0, kMsWidth * 8, st));
  const int xgrid = std::max(1, std::min<int>(g->num_sms * 8, (int)((g->nv + 31) / 32)));
  ms_extract<OP><<<xgrid, 256, 0, st>>>(a, want_out ? b->d_out : nullptr, b->d_sums);
  THV_CUDA(cudaGetLastError());
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
                                  const thv_batch_opts *o, uint32_t *out, uint64_t *sums,
                                  thv_stats &acc) {
  std::vector<uint32_t> vals(g->nv);
  for (uint32_t i = 0; i < k; i++) {
    thv_run_opts ro{};
    ro.source = src[i];
    ro.timeout_ms = o ? o->timeout_ms : 0;
    thv_stats st1{};
    THV_TRY(run_minprop(g, THV_ALGO_BFS, &ro, st, &st1));
    uint32_t *dst = out ? out + (uint64_t)i * g->nv : vals.data();
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

thv_status run_batch(thv_graph *g, thv_algo algo, const uint32_t *sources,
                     uint32_t n, const thv_batch_opts *o, uint32_t *out,
                     uint64_t *checksums, thv_stats *stats) {
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
  uint32_t small = 64, chunk = 256;
  if (o && o->small_degree) small = o->small_degree;
  if (o && o->chunk_edges) chunk = std::max<uint32_t>(32, (o->chunk_edges + 31) / 32 * 32);
  THV_TRY(ensure_batch_state(g, sssp, chunk, small, out != nullptr));
  BatchState *b = g->bs;
  cudaStream_t st = o && o->stream ? (cudaStream_t)o->stream : g->stream;
  MsArgs a{};
  a.off = g->d_off;
  a.blk_vb = g->plan.d_vbegin;
  a.blk_base = g->plan.d_base;
  a.host_base = g->h_edges_dev;
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
  a.cap_s = b->cap_s;
  a.cap_b = b->cap_b;
  a.ctrl = b->d_ctrl;
  a.sources = b->d_sources;
  const uint32_t tmo = o && o->timeout_ms ? o->timeout_ms : 60000u;
  a.timeout_ns = (unsigned long long)tmo * 1000000ull;
  a.nblk = (uint32_t)g->plan.blocks.size();
  a.nv = (uint32_t)g->nv;
  a.ngroups = b->ngroups;
  a.max_iters = (uint32_t)std::min<uint64_t>(g->nv + 2, 0x7FFFFFF0ull) * 2 + 8;
  a.small_deg = small;
  a.chunk = chunk;
  a.delta = o && o->sssp_delta ? o->sssp_delta : 2u;
  thv_stats local{};
  uint32_t launches = 0;
  float dev_ms = 0.f;
  for (uint32_t first = 0; first < n; first += group) {
    const uint32_t k = std::min(group, n - first);
    a.k = k;
    memcpy(b->h_sources, sources + first, k * 4);
    THV_CUDA(cudaEventRecord(b->ev0, st));
    thv_status s = g->esz == 8
        ? (sssp ? launch_group<MS_SSSP, 8>(g, a, st, out != nullptr, launches)
                : launch_group<MS_BFS, 8>(g, a, st, out != nullptr, launches))
        : (sssp ? fail(THV_EINVAL, "SSSP needs 8-byte weighted edges")
                : launch_group<MS_BFS, 4>(g, a, st, out != nullptr, launches));
    if (s != THV_OK) return s;
    THV_CUDA(cudaEventRecord(b->ev1, st));
    THV_CUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, sizeof(MsCtrl), cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaMemcpyAsync(b->h_sums, b->d_sums, kMsWidth * 8, cudaMemcpyDeviceToHost, st));
    if (out)
      THV_CUDA(cudaMemcpyAsync(out + (uint64_t)first * g->nv, b->d_out, (uint64_t)k * g->nv * 4,
                               cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaStreamSynchronize(st));
    float ms_ = 0.f;
    cudaEventElapsedTime(&ms_, b->ev0, b->ev1);
    dev_ms += ms_;
    const MsCtrl &hc = *b->h_ctrl;
    if (hc.err == kDevErrDepth) {
      // deeper than the u8 level bytes hold: run this group one source at a time
      THV_TRY(fallback_single(g, sources + first, k, st, o, out ? out + (uint64_t)first * g->nv : nullptr,
                              checksums ? checksums + first : nullptr, local));
      continue;
    }
    if (hc.err == kDevErrBarrier) return fail(THV_ETIMEOUT, "grid barrier wait exceeded %u ms", tmo);
    if (hc.err == kDevErrIters) return fail(THV_ETIMEOUT, "iteration cap reached");
    if (hc.err) return fail(THV_EDEVICE, "batch device error %u", hc.err);
    if (checksums) memcpy(checksums + first, b->h_sums, k * 8);
    local.iterations += hc.iters;
    local.edges_expanded += hc.edges;
    local.hbm_edge_bytes += hc.hbm_bytes;
    local.link_edge_bytes += hc.link_bytes;
    local.h2d_bytes += kMsWidth * 4;
    local.d2h_bytes += sizeof(MsCtrl) + kMsWidth * 8 + (out ? (uint64_t)k * g->nv * 4 : 0);
  }
  local.device_ms = dev_ms;
  local.kernel_launches = launches;
  local.wall_ms = now_ms() - t0;
  if (stats) *stats = local;
  return THV_OK;
}

}  // namespace thv
