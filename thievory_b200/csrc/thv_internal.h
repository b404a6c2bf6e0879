// Internal host-side definitions shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "thv.h"

namespace thv {

// Thread-local error message; returns the status for `return fail(...)`.
thv_status fail(thv_status s, const char *fmt, ...);
bool alloc_should_fail();  // host fault-injection hook

#define THV_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return ::thv::fail(THV_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__,     \
                         #call, cudaGetErrorString(e_));                    \
  } while (0)

#define THV_TRY(expr)                          \
  do {                                         \
    thv_status s_ = (expr);                    \
    if (s_ != THV_OK) return s_;               \
  } while (0)

// Device allocation with the fault-injection hook.
thv_status dev_alloc(void **p, size_t bytes, const char *what);
thv_status pinned_alloc(void **p, size_t bytes, const char *what);
void dev_free(void *p);
void pinned_free(void *p);

// Edge block: a vertex range whose adjacency is contiguous in the edge array.
struct Block {
  uint32_t vbegin, vend;
  uint64_t ebegin, eend;  // edge indices
  bool resident;
  uint64_t dev_elem;      // element offset inside the resident buffer
};

// Dense-iteration tile (PageRank): a vertex range with <= kTileEdges edges
// inside one block, or one part of a high-degree vertex ("split" tile).
struct __align__(16) PrTile {
  uint64_t ebegin, eend;
  uint32_t vbegin, vend;
  uint32_t block;
  uint32_t split;  // 0, or 1 + index of the split vertex
};

constexpr uint64_t kDefaultBlockBytes = 64ull << 20;  // reference PARTITION_SIZE_MB
constexpr size_t kEdgePad = 1024;                     // bytes of slack past arrays
constexpr uint32_t kDefaultListDeg = 64;  // small-list cache threshold (CSR/WCSR)
constexpr size_t kListLead = 128;         // slack before the first cached list

struct Plan {
  bool valid = false;
  uint64_t budget_bytes = 0, block_bytes = 0;
  uint32_t policy = 0;
  std::vector<Block> blocks;
  std::vector<uint32_t> vbegin;     // nb+1 entries
  std::vector<uint64_t> base;       // per-block virtual base address
  char *d_resident = nullptr;       // packed resident blocks
  size_t d_resident_bytes = 0;
  uint32_t *d_vbegin = nullptr;
  uint64_t *d_base = nullptr;
  uint64_t resident_edge_bytes = 0, host_edge_bytes = 0;
  // small-list cache: lists with 0 < deg < list_deg in host blocks, packed
  // in d_lists (element 0 at d_lists + kListLead); d_list_idx[v] = element
  // index of v's list
  uint32_t list_deg = 0;
  char *d_lists = nullptr;
  uint32_t *d_list_idx = nullptr;
  uint64_t list_bytes = 0, list_vertices = 0, d_lists_bytes = 0;
  // access tracking: link bytes per block (device counters) and the flags
  uint32_t flags = 0;
  unsigned long long *d_access = nullptr;
  // PageRank tiles (built lazily)
  bool tiles_valid = false;
  std::vector<PrTile> tiles;
  std::vector<uint32_t> split_parts;  // per split vertex
  PrTile *d_tiles = nullptr;
  uint32_t *d_split_parts = nullptr;
  uint64_t tiles_hbm_bytes = 0, tiles_link_bytes = 0;
};

// Small-list cache as the kernels see it: lists with 0 < deg < deg_lt whose
// block is read from the host are mirrored in HBM; idx[v] is the element
// index of v's list there (element 0 at base).  deg_lt = 0 disables it.
struct ListCache {
  const uint32_t *idx;
  unsigned long long base;
  uint32_t deg_lt, pad;
};

inline ListCache list_cache_of(const Plan &p) {
  ListCache c{nullptr, 0, 0, 0};
  if (p.list_deg && p.d_lists) {
    c.idx = p.d_list_idx;
    c.base = (unsigned long long)(p.d_lists + kListLead);
    c.deg_lt = p.list_deg;
  }
  return c;
}

struct MinState;  // minprop.cu
struct PrState;   // pagerank.cu
struct BatchState;  // batch.cu

}  // namespace thv

struct thv_graph {
  uint64_t nv = 0, ne = 0;
  thv_format fmt = THV_FMT_CSR;
  uint32_t esz = 4;       // bytes per edge in memory (host and HBM copies)
  bool weighted = false;
  bool sorted = false;     // every adjacency list ascending by neighbour id
  bool symmetric = false;  // every u->w has w->u (asserted or by construction)
  int64_t hub = -1;        // a vertex of maximum out-degree (lazily found)
  uint32_t hub_vertex() {
    if (hub < 0) {
      hub = 0;
      for (uint64_t v = 1; v < nv; v++)
        if (off[v + 1] - off[v] > off[hub + 1] - off[hub]) hub = (int64_t)v;
    }
    return (uint32_t)hub;
  }
  // packed weighted edges: 4 bytes = dst << wshift | (w - wbase)
  bool packed = false;
  uint32_t wshift = 0, wbase = 0;
  int device = 0;
  // host
  std::vector<uint64_t> off;      // nv+1
  void *h_edges = nullptr;        // pinned + mapped, padded
  size_t h_edges_bytes = 0;
  uint64_t h_edges_dev = 0;       // device address of h_edges
  std::vector<uint32_t> outdeg;   // CSC only
  mutable std::vector<uint32_t> h_unpacked;  // {dst, w} view of packed edges
  // link bytes recorded under earlier tracked plans, per vertex range
  // (access_vb has one entry more than access_bytes)
  std::vector<uint32_t> access_vb;
  std::vector<uint64_t> access_bytes;
  // device
  cudaStream_t stream = nullptr;
  uint64_t *d_off = nullptr;
  uint32_t *d_outdeg = nullptr;   // CSC only
  int num_sms = 0;
  thv::Plan plan;
  thv::MinState *ms = nullptr;
  thv::PrState *ps = nullptr;
  uint64_t *d_in_off = nullptr;   // in-edge transpose (direction-optimising BFS)
  uint32_t *d_in_adj = nullptr;
  bool in_valid = false;
  thv::BatchState *bs = nullptr;              // state of the batched run in progress
  thv::BatchState *bs_keep[2] = {nullptr, nullptr};  // kept per algorithm: BFS, SSSP
  // last run
  int last_algo = -1;
  size_t device_bytes = 0;
};

namespace thv {


thv_status graph_init_device(thv_graph *g);  // stream, d_off, d_outdeg
thv_status set_packing(thv_graph *g, bool on);  // weighted graphs only
thv_status replan_by_access(thv_graph *g);      // THV_PLACE_ACCESS, same budget
thv_status ensure_transpose(thv_graph *g, cudaStream_t st);  // transpose.cu
thv_status convert_edge_list(const char *txt, const char *out_path, thv_format fmt,
                             uint32_t skip, uint32_t flags, int device, uint64_t *nv_out,
                             uint64_t *ne_out);  // convert.cu
void transpose_free(thv_graph *g);
thv_status ensure_plan(thv_graph *g);
thv_status build_tiles(thv_graph *g);
void plan_free(thv_graph *g);

thv_status run_minprop(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                       cudaStream_t st, thv_stats *stats);
thv_status minprop_values(thv_graph *g, uint32_t *out, cudaStream_t st);
const uint32_t *minprop_device_values(thv_graph *g);
void minprop_free(thv_graph *g);

thv_status run_pagerank(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                        cudaStream_t st, thv_stats *stats);
thv_status pagerank_values(thv_graph *g, double *out, cudaStream_t st);
void pagerank_free(thv_graph *g);

thv_status run_batch(thv_graph *g, thv_algo algo, const uint32_t *sources,
                     uint32_t n, const thv_batch_opts *o, uint32_t *out,
                     uint64_t *checksums, thv_stats *stats);
thv_status run_batch_rows(thv_graph *g, thv_algo algo, const uint32_t *sources,
                          uint32_t n, const thv_batch_opts *o, uint32_t *const *rows,
                          uint64_t *checksums, thv_stats *stats);
void batch_free(thv_graph *g);
thv_status batch_config(thv_graph *g, thv_algo algo, thv_batch_config *out);

// Continuous batched group of the server (batch.cu): up to 64 sources of
// one algorithm share a traversal that stays on the device; between
// launches, sources whose pending set is empty retire (live_collect) and
// new ones join free mask bits (live_add), each keeping its single-source
// encoding relative to its own start (base).
struct LiveGroup {
  bool sssp = false, running = false;
  uint32_t small = 64, chunk = 256, threads = 512;  // launch configuration
  uint32_t mid = 64, gsmall = 32, gmid = 4;
  uint32_t iter = 0, level = 1, thr = 0, width = 0;  // where the next launch resumes
  unsigned long long active = 0;                     // mask bits in use
  uint32_t base[64] = {};  // per bit: BFS level byte / SSSP distance of its source vertex
  uint32_t *d_buf = nullptr, *h_buf = nullptr;       // 4 x 64 u32 staging
  unsigned long long *d_sums = nullptr, *h_sums = nullptr;
  uint64_t edges = 0, hbm_bytes = 0, link_bytes = 0;  // since the group started
  BatchState *bs = nullptr;  // the group's own traversal state
};
thv_status live_open(thv_graph *g, LiveGroup *lg, bool sssp);
void live_close(LiveGroup *lg);
// Whether a running group can take another source (free bit, BFS level and
// SSSP distance headroom); a group that is not running always can.
bool live_can_join(const thv_graph *g, const LiveGroup *lg);
// Adds k sources (a fresh traversal if the group is not running); bits[t]
// receives the mask bit of sources[t].
thv_status live_add(thv_graph *g, LiveGroup *lg, uint32_t k, const uint32_t *sources,
                    uint32_t *bits, uint32_t timeout_ms, cudaStream_t st);
// Runs up to `iters` iterations; *finished = bits whose sources are done;
// *too_deep when a BFS level left the u8 range (the group must be dropped).
thv_status live_step(thv_graph *g, LiveGroup *lg, uint32_t iters, uint32_t timeout_ms,
                     cudaStream_t st, unsigned long long *finished, bool *too_deep);
// Checksums (sums[bit]) and, where out[bit] is set, values of the finished
// bits (via the device buffer d_stage of nv u32); frees the bits.
thv_status live_collect(thv_graph *g, LiveGroup *lg, unsigned long long fin, uint64_t *sums,
                        uint32_t *const *out, uint32_t *d_stage, cudaStream_t st);

thv_status generate_rmat(const thv_rmat_opts *o, thv_format fmt, int device,
                         thv_graph **out);

double now_ms();

}  // namespace thv
