/*
 * thv_oracle.h -- CPU oracle for the Thievory frontier engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: the GPU engine in
 * thievory_b200/ never links, calls or loads anything declared here.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm use it.
 *
 * It restates, on the CPU, what the reference computes on the GPU:
 *   - value encoding of src/graph.cuh:244-265 (BFS/SSSP: source = 1,
 *     unreached = n+1; CC: label starts at the vertex id);
 *   - BFS relaxation of src/bfs/bfs_kernels.cu:4-76 (level + 1, atomicMin);
 *   - CC min-label push of src/cc/cc_kernels.cu:4-68;
 *   - SSSP relaxation of src/sssp/sssp_kernels.cu:106-144 with the real edge
 *     weights (the reference's own weights are defective: it adds a constant
 *     20 on resident edges and reads an unwritten array elsewhere);
 *   - PageRank as the fixed-iteration, dangling-redistributing power method
 *     (damping 0.85, 20 iterations, FP64), which differs on purpose from the
 *     tolerance-driven variants in src/pr/pr_kernels.cu:449-476 / :846-860;
 *   - the byte formats written by converter/converter.cpp:483-589 (.csc),
 *     :676-774 (.csr) and :775-805 (.wcsr), and the headerless values.bin of
 *     src/graph.cuh:817-852.
 *
 * Graph generation (seeded RMAT, dedup, self-loop removal, id permutation,
 * weights) is defined here; the GPU generator in the engine must reproduce it
 * byte for byte.
 */
#ifndef THV_ORACLE_H
#define THV_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counter-based RNG (splitmix64 finaliser, Steele/Lea/Flood 2014) ---- */
uint64_t thvo_mix64(uint64_t x);

/* RMAT quadrant thresholds as 32-bit integers: floor(p * 2^32). */
void thvo_rmat_thresholds(double a, double b, double c, uint32_t out[3]);

/* Seeded bijection on [0, 2^scale) used to scatter RMAT hub ids. */
uint64_t thvo_permute(uint64_t x, uint32_t scale, uint64_t seed);

/* Edge weight in [1,64] as a function of the (src,dst) pair only. */
uint32_t thvo_weight(uint64_t seed, uint32_t src, uint32_t dst);

/* Raw RMAT edges i in [first, first+count): permuted ids, self-loops kept. */
void thvo_rmat_edges(uint32_t scale, uint64_t seed, const uint32_t thr[3],
                     uint64_t first, uint64_t count, uint32_t *src,
                     uint32_t *dst);

/*
 * Build a deduplicated, self-loop-free CSR sorted by (src,dst) from an edge
 * list.  off has nv+1 entries.  *adj is malloc'd; *ne receives its length.
 * If symmetric != 0 every edge is also inserted reversed first.
 */
int thvo_build_csr(uint64_t nv, uint64_t n_raw, const uint32_t *src,
                   const uint32_t *dst, int symmetric, uint64_t *off,
                   uint32_t **adj, uint64_t *ne);

/* Full generator: nv = 2^scale, E_gen = edge_factor * nv. */
int thvo_generate(uint32_t scale, uint32_t edge_factor, uint64_t seed,
                  double a, double b, double c, int symmetric, uint64_t *off,
                  uint32_t **adj, uint64_t *ne);

/* Weights for a CSR: w[i] = thvo_weight(seed, src(i), adj[i]). */
void thvo_weights(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  uint64_t seed, uint32_t *w);

/* CSR (out-edges) -> CSC (in-edges sorted by (dst,src)) + out-degrees. */
void thvo_transpose(uint64_t nv, uint64_t ne, const uint64_t *off,
                    const uint32_t *adj, uint64_t *in_off, uint32_t *in_adj,
                    uint32_t *outdeg);

/* n sources drawn uniformly (seeded) from vertices with out-degree > 0. */
int thvo_sources(uint64_t nv, const uint64_t *off, uint64_t seed, uint32_t n,
                 uint32_t *out);

/* ---- algorithms (value encoding of the reference) ---- */
/* adj_stride: 1 for 4-byte edges, 2 for interleaved {dst,w} 8-byte edges. */
int thvo_bfs(uint64_t nv, const uint64_t *off, const uint32_t *adj,
             uint32_t adj_stride, uint32_t src, uint32_t *level);
int thvo_bfs_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                 uint32_t adj_stride, uint32_t src, uint32_t *level);
int thvo_cc(uint64_t nv, const uint64_t *off, const uint32_t *adj,
            uint32_t adj_stride, uint32_t *label);
int thvo_cc_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                uint32_t adj_stride, uint32_t *label);
/* Weighted: interleaved {dst,w} (wadj, stride 2) or split adj + w arrays. */
int thvo_sssp(uint64_t nv, const uint64_t *off, const uint32_t *adj,
              const uint32_t *w, uint32_t stride, uint32_t src,
              uint32_t *dist);
int thvo_sssp_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  const uint32_t *w, uint32_t stride, uint32_t src,
                  uint32_t *dist);
/* PageRank over out-edges (CSR). */
int thvo_pagerank(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  uint32_t adj_stride, uint32_t iters, double damping,
                  double *rank);
/* PageRank over in-edges (CSC) with explicit out-degrees. */
int thvo_pagerank_csc(uint64_t nv, const uint64_t *in_off,
                      const uint32_t *in_adj, const uint32_t *outdeg,
                      uint32_t iters, double damping, double *rank);

/* PageRank with the reference engine's own semantics (FP64 values, rounds
 * until no vertex changes by more than its tolerance, no dangling
 * redistribution).  pull: in-edges (CSC) with explicit out-degrees;
 * push: out-edges (CSR, residual form).  *rounds gets the number of rounds;
 * returns -2 when max_rounds ran out. */
int thvo_pagerank_ref_pull(uint64_t nv, const uint64_t *in_off,
                           const uint32_t *in_adj, const uint32_t *outdeg,
                           uint32_t max_rounds, double *rank, uint32_t *rounds);
int thvo_pagerank_ref_push(uint64_t nv, const uint64_t *off,
                           const uint32_t *adj, uint32_t adj_stride,
                           uint32_t max_rounds, double *rank, uint32_t *rounds);

/* Sum of out-degrees of vertices with value < nv+1 (edges a single-source
 * traversal must expand: the GTEPS numerator). */
uint64_t thvo_reached_edges(uint64_t nv, const uint64_t *off,
                            const uint32_t *val);

/* ---- files (converter byte formats) ---- */
/* .csr: u64 nv, u64 ne, u64 off[nv], u32 adj[ne], u32 w[ne] (w may be NULL:
 * the converter's default weight 20 is written). */
int thvo_write_csr(const char *path, uint64_t nv, uint64_t ne,
                   const uint64_t *off, const uint32_t *adj,
                   const uint32_t *w);
/* .csc: u64 nv, u64 ne, u64 in_off[nv], u32 in_adj[ne], u32 outdeg[nv]. */
int thvo_write_csc(const char *path, uint64_t nv, uint64_t ne,
                   const uint64_t *in_off, const uint32_t *in_adj,
                   const uint32_t *outdeg);
/* .wcsr: u64 nv, u64 ne, u64 off[nv], {u32 dst, u32 w}[ne]. */
int thvo_write_wcsr(const char *path, uint64_t nv, uint64_t ne,
                    const uint64_t *off, const uint32_t *adj,
                    const uint32_t *w);
int thvo_write_values(const char *path, const void *vals, uint64_t n,
                      uint32_t elem_size);

/* Wall-clock seconds (monotonic). */
double thvo_now(void);
/* Threads OpenMP will use. */
int thvo_threads(void);
void thvo_set_threads(int n); /* OpenMP threads for later calls */

#ifdef __cplusplus
}
#endif
#endif
