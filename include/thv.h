/*
 * thv.h -- C ABI of the B200 out-of-memory graph engine (thievory_b200).
 *
 * Plain C, no CUDA or torch types: the CLI (`./main`), the Python host mirror
 * (thievory_b200/__init__.py, via ctypes), tests and bench.py all call these.
 *
 * Conventions
 *   - Every call returns thv_status; the library never calls exit() and never
 *     lets a C++ exception cross this boundary.  thv_last_error() gives a
 *     thread-local message for the last failing call on that thread.
 *   - The caller owns output buffers; the library owns device memory and the
 *     pinned host copy of the edges.
 *   - A thv_graph is used by one host thread at a time.  The serving API
 *     (thv_serve_*) is internally multi-threaded and may be called from any
 *     thread.
 *
 * Reference interfaces replaced (paths inside qqueke/Thievory):
 *   thv_open / thv_close        CSR<E>::ReadInputFile  src/graph.cuh:641-815,
 *                               CSR<E>::Free           src/graph.cuh:855-923
 *   thv_plan                    CSR<E>::InitData / SetPartitionsConfig /
 *                               SetNumStaticEdges      src/graph.cuh:270-638
 *   thv_run                     BFS32 src/bfs/bfs.cu:8, CC32 src/cc/cc.cu:71,
 *                               SSSP32 src/sssp/sssp.cu:10, PR32 src/pr/pr.cu:11,
 *                               PR32_PUSH src/pr/pr.cu:1030
 *   thv_values / thv_write_values
 *                               CSR<E>::DumpValues     src/graph.cuh:817-852
 *   thv_save                    converter/converter.cpp:483-589 (.csc),
 *                               :676-774 (.csr), :775-805 (.wcsr)
 *   thv_batch_run, thv_batch_tuned, thv_serve_*, thv_generate_rmat
 *                               no counterpart in the reference (new surface)
 */
#ifndef THV_H
#define THV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define THV_ABI_VERSION 4

typedef enum thv_status {
  THV_OK = 0,
  THV_EINVAL = 1,       /* bad argument (null pointer, source >= n, ...) */
  THV_EIO = 2,          /* file cannot be opened, read or written */
  THV_EFORMAT = 3,      /* truncated or malformed graph file */
  THV_ENOMEM = 4,       /* device / pinned allocation failed, or over budget */
  THV_ECUDA = 5,        /* CUDA runtime error (message in thv_last_error) */
  THV_ETIMEOUT = 6,     /* a bounded device wait or iteration cap ran out */
  THV_EUNSUPPORTED = 7, /* option combination not supported */
  THV_EBUSY = 8,        /* serving: queue full / not admitted */
  THV_ENOTREADY = 9,    /* serving: result not ready yet */
  THV_EDEVICE = 10      /* kernel reported an internal error (queue overflow) */
} thv_status;

/* File / in-memory layouts (converter byte formats). */
typedef enum thv_format {
  THV_FMT_CSR = 0,  /* u64 nv, u64 ne, u64 off[nv], u32 dst[ne], u32 w[ne] */
  THV_FMT_CSC = 1,  /* u64 nv, u64 ne, u64 in_off[nv], u32 src[ne], u32 outdeg[nv] */
  THV_FMT_WCSR = 2  /* u64 nv, u64 ne, u64 off[nv], {u32 dst, u32 w}[ne] */
} thv_format;

/* thv_open flags */
#define THV_OPEN_WEIGHTS 1u /* CSR: load the trailing weight section (SSSP) */

typedef enum thv_algo {
  THV_ALGO_BFS = 0,     /* u32 levels: source 1, unreached n+1 */
  THV_ALGO_CC = 1,      /* u32 labels: min id of any vertex reaching v */
  THV_ALGO_SSSP = 2,    /* u32: min(distance + 1, n+1); needs weights */
  THV_ALGO_PR_PUSH = 3, /* double ranks (FP32 on device); CSR input */
  THV_ALGO_PR_PULL = 4  /* double ranks (FP32 on device); CSC input */
} thv_algo;

typedef struct thv_graph thv_graph;

/* ---- graphs ---- */
thv_status thv_open(const char *path, thv_format fmt, uint32_t flags,
                    int device, thv_graph **out);

/* Build from host arrays (copied).  off has nv+1 entries (off[nv] = ne).
 * edges: u32 ids (esz 4) or interleaved {dst,w} pairs (esz 8, WCSR).
 * outdeg: required for THV_FMT_CSC (in-edge graphs), else NULL. */
thv_status thv_from_arrays(uint64_t nv, uint64_t ne, const uint64_t *off,
                           const void *edges, uint32_t esz, thv_format fmt,
                           const uint32_t *outdeg, int device,
                           thv_graph **out);

typedef struct thv_rmat_opts {
  uint32_t scale;       /* nv = 2^scale */
  uint32_t edge_factor; /* raw edges = edge_factor * nv (before dedup) */
  uint64_t seed;
  double a, b, c;       /* quadrant probabilities (d = 1 - a - b - c) */
  uint32_t symmetric;   /* insert every edge both ways (CC) */
  uint32_t pad;
} thv_rmat_opts;

/* Seeded RMAT on the GPU: self-loops and duplicates removed, ids permuted,
 * CSR sorted by (src,dst); WCSR adds weights in [1,64]; CSC is the transpose
 * with out-degrees.  Byte-identical to the CPU oracle's generator. */
thv_status thv_generate_rmat(const thv_rmat_opts *o, thv_format fmt,
                             int device, thv_graph **out);

thv_status thv_save(const thv_graph *g, const char *path);

/* Text edge list -> .csr / .csc / .wcsr, sorting on the GPU; the bytes of
 * converter/converter.cpp (ConvertTxtToBCSR :676-808, ConvertTxtToBCSC
 * :483-589).  The first skip_lines lines are dropped; each later line is
 * "src dst [w]" (w read with THV_CONVERT_WEIGHTED, else 20); a field that
 * does not parse keeps the previous line's value, as the converter's
 * stream does.  Duplicates and self-loops are kept; nv = max id + 1.
 * nv_out / ne_out may be NULL. */
#define THV_CONVERT_WEIGHTED 1u   /* third column is the weight (-DWEIGHTED) */
#define THV_CONVERT_UNDIRECTED 2u /* add dst -> src for every line (-DUNDIRECTED) */
thv_status thv_convert(const char *txt_path, const char *out_path, thv_format fmt,
                       uint32_t skip_lines, uint32_t flags, int device,
                       uint64_t *nv_out, uint64_t *ne_out);
thv_status thv_close(thv_graph *g);

typedef struct thv_graph_info {
  uint64_t nv, ne;
  uint32_t fmt, esz;    /* edge size of the format: 8 for weighted, else 4 */
  uint32_t device, weighted;
  uint32_t mem_esz;     /* bytes per edge as stored (host and HBM): 4 when packed */
  uint32_t weight_bits; /* packed: low bits of an edge hold w - min weight; 0 = not packed */
  uint32_t sorted;      /* every list ascending by neighbour id */
  uint32_t symmetric;   /* marked symmetric (see thv_set_symmetric) */
} thv_graph_info;
thv_status thv_info(const thv_graph *g, thv_graph_info *out);
/* Weighted graphs are stored packed by default: each {u32 dst, u32 w} pair
 * becomes one u32, dst << b | (w - min w), whenever the id bits plus the
 * weight-range bits fit 32 bits (lossless; halves the edge bytes moved).
 * packed = 0 restores {dst, w} pairs, 1 packs again.  Drops the plan;
 * no effect on unweighted graphs. */
thv_status thv_set_edge_packing(thv_graph *g, int packed);
/* Asserts (1) or withdraws (0) that every edge u->w has its reverse w->u.
 * CC then runs as sampling union-find (THV_RUN_LABEL_PROPAGATION).
 * On a graph that is not symmetric, CC with this set returns the labels of
 * its weakly connected components instead of the reference's. */
thv_status thv_set_symmetric(thv_graph *g, int symmetric);
/* Host views of the graph (valid until thv_close); edges in the format's
 * layout ({dst, w} pairs for weighted graphs, unpacked on first use).
 * outdeg NULL unless CSC. */
thv_status thv_host_arrays(const thv_graph *g, const uint64_t **off,
                           const void **edges, const uint32_t **outdeg);

/* ---- placement plan (static HBM budget) ---- */
#define THV_PLACE_DENSEST 0u /* resident blocks chosen by edges per vertex */
#define THV_PLACE_PREFIX 1u  /* longest prefix of blocks (reference order) */
#define THV_PLACE_ACCESS 2u  /* blocks whose adjacency was read the most per
                                byte under earlier tracked plans first (then
                                densest) */

typedef struct thv_plan_opts {
  uint64_t hbm_budget_bytes; /* resident edge bytes; UINT64_MAX = all that fit */
  uint64_t block_bytes;      /* edge block size; 0 = 64 MiB */
  uint32_t policy;
  /* Small-list cache: adjacency lists with 0 < degree < small_list_degree
   * that fall in host blocks are copied, packed, into HBM first (host reads
   * of short lists are bound by the link's request rate, not its bytes);
   * blocks fill the rest of the budget.  The threshold is lowered until
   * the lists fit the budget.  BFS/CC/SSSP and the batched and served runs
   * read the cache; PageRank reads whole blocks and ignores it.
   * 0 = default (64 for CSR/WCSR, off for CSC); 1 = off. */
  uint32_t small_list_degree;
  uint32_t flags; /* THV_PLAN_* */
  uint32_t pad;
} thv_plan_opts;

/* thv_plan_opts.flags: count, per block, the adjacency bytes the traversal
 * kernels read from it, resident or over the link (thv_get_block_access);
 * the counts carry over to later plans of the graph for THV_PLACE_ACCESS.  Replaces
 * the reference's lazy caching of filtered partitions (src/bfs/bfs.cu:
 * 155-519) with measured, explicit re-placement. */
#define THV_PLAN_TRACK_ACCESS 1u

typedef struct thv_plan_info {
  uint64_t num_blocks, resident_blocks;
  uint64_t resident_edge_bytes, host_edge_bytes; /* resident includes the cache */
  uint64_t device_bytes; /* all device memory the graph holds */
  uint64_t small_list_degree; /* effective threshold; 0 = no cache */
  uint64_t small_list_bytes, small_list_vertices;
} thv_plan_info;

thv_status thv_plan(thv_graph *g, const thv_plan_opts *o); /* NULL = defaults */
thv_status thv_get_plan(const thv_graph *g, thv_plan_info *out);
/* Block table of the current plan: vbegin[0..nb] (first vertex of each
 * block, vbegin[nb] = nv) and resident[0..nb-1] (1 = held in HBM).  cap is
 * the capacity of resident (vbegin needs cap + 1); *nb receives the count. */
thv_status thv_get_blocks(const thv_graph *g, uint64_t cap, uint32_t *vbegin,
                          uint8_t *resident, uint64_t *nb);
/* Adjacency bytes read from each block since this plan was made, from HBM
 * or over the link (tracked plans).  bytes has cap entries. */
thv_status thv_get_block_access(const thv_graph *g, uint64_t cap, uint64_t *bytes,
                                uint64_t *nb);
/* Plan persistence: the block split, the resident set, the small-list
 * threshold and the access counts.  Loading re-creates exactly that plan
 * on the same graph (same vertex, edge and stored-edge sizes; otherwise
 * THV_EINVAL) and keeps the counts for THV_PLACE_ACCESS. */
thv_status thv_save_plan(const thv_graph *g, const char *path);
thv_status thv_load_plan(thv_graph *g, const char *path);

/* ---- single-source / whole-graph runs ---- */
typedef struct thv_run_opts {
  uint32_t source;       /* BFS / SSSP */
  uint32_t pr_iters;     /* 0 = 20 */
  double pr_damping;     /* 0 = 0.85 */
  uint32_t sssp_delta;   /* SSSP near/far window (0 = 8); CC initial label
                            window (0 = 1) */
  uint32_t timeout_ms;   /* bound on any device-side wait; 0 = 60000 */
  void *stream;          /* cudaStream_t to launch on; NULL = graph's own */
  uint32_t small_degree; /* expansion tuning; 0 = default */
  uint32_t chunk_edges;  /* expansion tuning; 0 = default */
  uint32_t flags;        /* THV_RUN_* */
  uint32_t sssp_growth;  /* SSSP window width factor per advance: 0 = 32,
                            1 = fixed windows (plain near/far) */
} thv_run_opts;

/* thv_run_opts.flags: also compute stats->checksum = sum over v of
 * splitmix64((v << 32) | value) (BFS/CC/SSSP), after the timed traversal */
#define THV_RUN_CHECKSUM 1u
/* BFS/CC/SSSP work-queue construction; same results either way.  Scan:
 * rebuild the queue from the pending bitmap every iteration (sorted vertex
 * order, two grid barriers per iteration; the default for BFS and CC).
 * Queue: queue vertices as they are lowered, scanning only when the near
 * window empties (one barrier per iteration; the default for SSSP). */
#define THV_RUN_SCAN_COMPACTION 2u
#define THV_RUN_QUEUE_COMPACTION 4u
/* BFS on a graph whose out-edges are all resident switches to bottom-up
 * levels over an in-edge transpose (built in HBM on first use) when the
 * frontier is large; this flag keeps every level top-down.  Same results. */
#define THV_RUN_TOP_DOWN_ONLY 8u
/* CC on a graph marked symmetric (thv_set_symmetric, or generated with
 * symmetric = 1) runs as sampling union-find, which reads the first two
 * neighbours of every vertex and the lists of vertices outside the largest
 * component only; this flag keeps min-label propagation.  Same labels. */
#define THV_RUN_LABEL_PROPAGATION 16u
/* PageRank with the reference engine's semantics instead of the
 * fixed-iteration FP32 method: FP64 values, no dangling redistribution,
 * rounds until no vertex changes by more than 1e-3.  Pull: r0 = 1/N,
 * r = 0.15 + 0.85 * sum of r(u)/outdeg(u) over in-edges, recomputed only
 * for vertices still active.  Push: residual form, r0 = 0.15.  Values agree
 * with the reference's to its comparer's 1e-3 absolute tolerance (its FP64
 * atomics make its own sums order-dependent).  pr_iters caps the rounds
 * (0 = 100000; THV_ETIMEOUT when reached); stats->iterations = rounds. */
#define THV_RUN_PR_REFERENCE 32u

typedef struct thv_stats {
  double device_ms;         /* CUDA-event time of the traversal */
  double wall_ms;           /* host time of the whole call */
  uint64_t iterations;
  uint64_t edges_expanded;  /* adjacency entries actually scanned */
  uint64_t hbm_edge_bytes;  /* adjacency bytes read from resident blocks */
  uint64_t link_edge_bytes; /* adjacency bytes read over the host link */
  uint64_t h2d_bytes;       /* explicit host->device copies in the call */
  uint64_t d2h_bytes;       /* explicit device->host copies in the call */
  uint32_t kernel_launches;
  uint32_t bottom_up_levels; /* BFS levels run bottom-up */
  uint64_t checksum;        /* with THV_RUN_CHECKSUM */
} thv_stats;

/* Runs algo.  out_values (host, may be NULL) receives u32[nv] or double[nv]
 * (PR).  stats may be NULL.  Synchronous. */
thv_status thv_run(thv_graph *g, thv_algo algo, const thv_run_opts *o,
                   void *out_values, thv_stats *stats);
/* Copy the last run's values (u32[nv], or double[nv] for PR) to the host. */
thv_status thv_values(thv_graph *g, void *out_values);
/* Write values as the reference does (headerless raw array). */
thv_status thv_write_values(const char *path, const void *values, uint64_t n,
                            uint32_t elem_size);

/* ---- batched multi-source BFS / SSSP ---- */
typedef struct thv_batch_opts {
  uint32_t group;        /* sources per group, 1..64; 0 = 64 */
  uint32_t timeout_ms;   /* 0 = 60000 */
  void *stream;
  uint32_t small_degree; /* expansion tuning; 0 = autotuned / default */
  uint32_t chunk_edges;  /* expansion tuning; 0 = autotuned / default */
  uint32_t sssp_delta;   /* shared near/far width for SSSP; 0 = 256 */
  uint32_t tune;         /* 1: without small_degree/chunk_edges, time the
                            first group under each candidate launch
                            configuration and keep the fastest (cached per
                            graph shape in memory and in $THV_TUNE_CACHE or
                            ~/.cache/thievory_b200_batch_tune.txt) */
  uint32_t sssp_growth;  /* SSSP window width factor per advance; 0 = default */
  /* Degree buckets of the expansion.  Vertices of out-degree below
   * small_degree go in groups of small_group per warp, those below
   * mid_degree in groups of mid_group per warp (a group's warp spreads the
   * group's edges over its 32 lanes), the rest in chunks of chunk_edges
   * edges per warp.  Any of small_degree, chunk_edges, mid_degree,
   * small_group, mid_group non-zero selects an explicit configuration (the
   * zeros among them take the defaults: mid_degree = small_degree, i.e. no
   * middle bucket; small_group 32; mid_group 4); all zero selects the tuned
   * or default one. */
  uint32_t mid_degree;
  uint32_t small_group;  /* 1..32 */
  uint32_t mid_group;    /* 1..32 */
  uint32_t pad;
} thv_batch_opts;

/* The batch kernel's launch configuration for a graph and algorithm: the
 * autotuned one when thv_batch_run with tune = 1 has timed it for a graph of
 * this shape (tuned = 1), else the default (tuned = 0). */
typedef struct thv_batch_config {
  uint32_t small_degree, mid_degree, chunk_edges, threads;
  uint32_t small_group, mid_group;
  uint32_t tuned, pad;
} thv_batch_config;

thv_status thv_batch_tuned(thv_graph *g, thv_algo algo, thv_batch_config *out);

/* Runs n sources in groups sharing one traversal each.  out (host, may be
 * NULL): n x nv u32, row i = values for sources[i] in the single-source
 * encoding, bit-exact equal to thv_run of that source.  checksums (may be
 * NULL): per source, sum over v of splitmix64((v << 32) | value) mod 2^64,
 * so results too large to copy can still be compared with single runs. */
thv_status thv_batch_run(thv_graph *g, thv_algo algo, const uint32_t *sources,
                         uint32_t n, const thv_batch_opts *o, uint32_t *out,
                         uint64_t *checksums, thv_stats *stats);

/* ---- serving (continuous batching) ---- */
/* A server owns the graph while it runs (no other thv_run on it meanwhile).
 * By default queries run in batched groups, one per algorithm, that stay on
 * the device: a query that arrives while its algorithm's group runs joins a
 * free source bit of it at the next iteration boundary, shares every later
 * edge read of that traversal, and leaves with its result as soon as its own
 * traversal is complete; the BFS and SSSP groups take turns.  An idle server
 * runs a lone query on the single-source kernel.  With group_min =
 * 0xFFFFFFFF, queries occupy slots of one resident traversal instead (u32
 * values per slot, admitted the same way).  Results are bit-identical to
 * thv_run of the same source. */
typedef struct thv_server thv_server;

typedef struct thv_serve_opts {
  uint32_t max_slots;        /* concurrent queries on the device, <= 64 */
  uint32_t queue_capacity;   /* waiting requests; 0 = 65536 */
  uint64_t mem_budget_bytes; /* device memory for per-query values (4 B per
                                vertex per slot); 0 = all slots */
  uint32_t timeout_ms;       /* bound on device waits; 0 = 60000 */
  uint32_t max_batch_iters;  /* slots: iterations per launch while requests
                                wait; batched groups: iterations per launch
                                while nothing waits and the other
                                algorithm's group is idle (else 1); 0 = 4 */
  uint32_t group_min;        /* batching: with nothing on the device, a
                                batched group of an algorithm starts when
                                at least group_min of its queries wait,
                                else the front query runs alone; a running
                                group admits every arrival of its algorithm
                                it has room for; 0 = measured defaults (BFS
                                4, SSSP 6); 0xFFFFFFFF = no batching
                                (slots) */
  uint32_t replan_every;     /* re-place the graph's blocks by measured
                                access (THV_PLACE_ACCESS, same budget) after
                                this many finished queries; 0 = never */
  uint32_t join_window;      /* batching: a running group admits arrivals
                                during its first join_window iterations
                                only (later ones start or wait for another
                                group); 0 = default (2); 0xFFFFFFFF = for
                                its whole life */
  uint32_t groups_per_algo;  /* batching: groups of one algorithm on the
                                device at once (1 or 2): with 2, a second
                                group starts for arrivals while the first
                                one drains (the two take turns); 0 = 1 */
} thv_serve_opts;

typedef struct thv_query_stats {
  double queue_ms;   /* submit -> admitted into a slot */
  double run_ms;     /* admitted -> result written */
  double latency_ms; /* submit -> result written */
  uint64_t checksum; /* sum over v of splitmix64((v << 32) | value) */
  uint32_t iterations;
  uint32_t slot;
  int32_t status;    /* thv_status of the query */
  uint32_t grouped;  /* 0: ran in a slot; 1: in a batched group (slot =
                        its mask bit); 2: alone on the single-source
                        kernel (the server was idle) */
  uint32_t joined;   /* 1: admitted into a group or slot traversal that was
                        already running on the device (it joined mid-flight
                        and shared that traversal's later iterations) */
  uint32_t pad;
} thv_query_stats;

thv_status thv_serve_start(thv_graph *g, const thv_serve_opts *o,
                           thv_server **out);
/* algo BFS or SSSP.  out_values (may be NULL): nv u32 written before the
 * ticket completes; it must stay valid until then.  Never blocks; THV_EBUSY
 * when the waiting queue is full. */
thv_status thv_serve_submit(thv_server *s, thv_algo algo, uint32_t source,
                            uint32_t *out_values, uint64_t *ticket);
/* THV_ENOTREADY until the query is done; then fills st and releases the
 * ticket. */
thv_status thv_serve_poll(thv_server *s, uint64_t ticket, thv_query_stats *st);
thv_status thv_serve_wait(thv_server *s, uint64_t ticket, thv_query_stats *st,
                          uint32_t timeout_ms);
/* Finishes every submitted query, then stops. */
thv_status thv_serve_stop(thv_server *s);

/* n sources drawn uniformly (seeded) from the vertices with out-degree > 0:
 * draw j tries splitmix64(key ^ (j << 24 | t)) mod nv for t = 0, 1, ... with
 * key = splitmix64(seed ^ 0x534F555243455331). */
thv_status thv_pick_sources(const thv_graph *g, uint64_t seed, uint32_t n,
                            uint32_t *out);

/* ---- allocation-free BFS ---- */
/* No counterpart in the reference: a BFS for callers that cannot allocate
 * device memory on this path (a host framework that owns all device memory
 * through its own pool, or a latency-critical path that cannot take
 * cudaMalloc's implicit device synchronisation).  Same kernel and results as
 * thv_run(THV_ALGO_BFS) -- u32 levels, source 1, unreached nv+1 -- over a
 * CSR the caller already holds in device (or host-mapped) memory: d_off
 * (nv+1 u64), d_adj (ne u32; 128-byte aligned, readable 16 bytes past its
 * end, as cudaMalloc allocations are) and the output d_values (nv u32).
 * It calls no allocator: its scratch is one 64 MiB static device array per
 * GPU, held until the process exits, so graphs whose scratch needs more
 * (about 16 bytes per vertex plus 0.3 bytes per edge) get THV_ENOMEM.  Calls
 * share that array: calls whose work overlaps on the GPU race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's address; make it before any stream capture.  That address is kept
 * for the life of the process: a cudaDeviceReset after the first call is not
 * supported.  stream: a cudaStream_t or NULL; iterations may be NULL.
 * Returns after the traversal has finished. */
thv_status thv_bfs_noalloc(const uint64_t *d_off, const uint32_t *d_adj,
                           uint64_t nv, uint64_t ne, uint32_t source,
                           uint32_t *d_values, void *stream,
                           uint64_t *iterations);

/* ---- misc ---- */
/* Host-link bandwidth of `device` in GB/s: a pinned cudaMemcpy host->device
 * of `bytes`, and a kernel streaming 16-byte zero-copy loads from pinned,
 * mapped host memory (the engine's non-resident edge path).  Either output
 * may be NULL. */
thv_status thv_link_bandwidth(int device, uint64_t bytes, double *memcpy_gbs,
                              double *zerocopy_gbs);
const char *thv_last_error(void);
const char *thv_status_str(thv_status s);
uint32_t thv_abi_version(void);
/* Host fault injection for tests: the n-th subsequent pinned/device
 * allocation made by the library fails (0 disables). */
void thv_debug_fail_alloc_after(uint32_t n);
/* Failure detection without a fault: a two-block launch in which one block
 * never reaches the grid barrier, so the other's bounded wait runs out after
 * timeout_ms (1..10000) and records the error the traversals report.
 * Returns THV_ETIMEOUT; the context stays usable. */
thv_status thv_debug_wait_timeout(int device, uint32_t timeout_ms);

#ifdef __cplusplus
}
#endif
#endif /* THV_H */
