/*
 * thv_oracle.c -- CPU oracle (test infrastructure; see thv_oracle.h).
 *
 * Plain C + OpenMP.  Every algorithm keeps the reference's value encoding
 * (src/graph.cuh:244-265): BFS/SSSP values are "distance + 1" with the source
 * at 1 and unreached vertices at n+1; CC labels start at the vertex id and
 * settle at the minimum id of any vertex that reaches them.
 */
#define _GNU_SOURCE
#include "thv_oracle.h"

#include <errno.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ RNG -- */

uint64_t thvo_mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

void thvo_rmat_thresholds(double a, double b, double c, uint32_t out[3]) {
  const double two32 = 4294967296.0;
  double ca = a, cb = a + b, cc = a + b + c;
  out[0] = ca >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(ca * two32);
  out[1] = cb >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(cb * two32);
  out[2] = cc >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(cc * two32);
}

#define THVO_PERM_SALT 0x5045524D55544531ull
#define THVO_WEIGHT_SALT 0x5745494748543634ull
#define THVO_SOURCE_SALT 0x534F555243455331ull

uint64_t thvo_permute(uint64_t x, uint32_t scale, uint64_t seed) {
  if (scale == 0) return 0;
  const uint64_t mask = scale >= 64 ? ~0ull : ((1ull << scale) - 1);
  const uint32_t h = (scale + 1) / 2;
  const uint64_t key = thvo_mix64(seed ^ THVO_PERM_SALT);
  for (uint64_t r = 0; r < 4; r++) {
    const uint64_t k = thvo_mix64(key + r);
    x = (x * (k | 1ull)) & mask; /* odd multiplier: bijective mod 2^scale */
    x ^= x >> h;                 /* xorshift: bijective on scale bits */
    x = (x + (k >> 17)) & mask;  /* offset: bijective mod 2^scale */
  }
  return x;
}

uint32_t thvo_weight(uint64_t seed, uint32_t src, uint32_t dst) {
  const uint64_t key = thvo_mix64(seed ^ THVO_WEIGHT_SALT);
  return 1u + (uint32_t)(thvo_mix64(key ^ (((uint64_t)src << 32) | dst)) & 63u);
}

void thvo_rmat_edges(uint32_t scale, uint64_t seed, const uint32_t thr[3],
                     uint64_t first, uint64_t count, uint32_t *src,
                     uint32_t *dst) {
  const uint64_t key = thvo_mix64(seed);
  const uint32_t words = (scale + 1) / 2;
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)count; j++) {
    const uint64_t i = first + (uint64_t)j;
    uint64_t u = 0, v = 0;
    for (uint32_t k = 0; k < words; k++) {
      const uint64_t x = thvo_mix64(key ^ ((i << 5) | k));
      for (uint32_t half = 0; half < 2; half++) {
        const uint32_t lvl = 2 * k + half;
        if (lvl >= scale) break;
        const uint32_t r = half ? (uint32_t)(x >> 32) : (uint32_t)x;
        uint32_t ub, vb;
        if (r < thr[0]) {
          ub = 0; vb = 0;
        } else if (r < thr[1]) {
          ub = 0; vb = 1;
        } else if (r < thr[2]) {
          ub = 1; vb = 0;
        } else {
          ub = 1; vb = 1;
        }
        u = (u << 1) | ub;
        v = (v << 1) | vb;
      }
    }
    src[j] = (uint32_t)thvo_permute(u, scale, seed);
    dst[j] = (uint32_t)thvo_permute(v, scale, seed);
  }
}

/* ------------------------------------------------------------- builders -- */

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

int thvo_build_csr(uint64_t nv, uint64_t n_raw, const uint32_t *src,
                   const uint32_t *dst, int symmetric, uint64_t *off,
                   uint32_t **adj_out, uint64_t *ne_out) {
  uint64_t *deg = (uint64_t *)calloc(nv + 1, sizeof(uint64_t));
  if (!deg) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n_raw; i++) {
    const uint32_t u = src[i], v = dst[i];
    if (u == v || u >= nv || v >= nv) continue;
#pragma omp atomic
    deg[u]++;
    if (symmetric) {
#pragma omp atomic
      deg[v]++;
    }
  }
  uint64_t *pos = (uint64_t *)malloc((nv + 1) * sizeof(uint64_t));
  if (!pos) { free(deg); return -1; }
  uint64_t acc = 0;
  for (uint64_t v = 0; v < nv; v++) { pos[v] = acc; acc += deg[v]; }
  pos[nv] = acc;
  uint32_t *tmp = (uint32_t *)malloc((acc + 1) * sizeof(uint32_t));
  uint64_t *fill = (uint64_t *)malloc((nv + 1) * sizeof(uint64_t));
  if (!tmp || !fill) { free(deg); free(pos); free(tmp); free(fill); return -1; }
  memcpy(fill, pos, (nv + 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n_raw; i++) {
    const uint32_t u = src[i], v = dst[i];
    if (u == v || u >= nv || v >= nv) continue;
    uint64_t p;
#pragma omp atomic capture
    p = fill[u]++;
    tmp[p] = v;
    if (symmetric) {
#pragma omp atomic capture
      p = fill[v]++;
      tmp[p] = u;
    }
  }
  free(fill);
  /* sort + dedup each adjacency in place, record new degrees */
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)nv; v++) {
    uint32_t *a = tmp + pos[v];
    const uint64_t d = pos[v + 1] - pos[v];
    if (d > 1) qsort(a, d, sizeof(uint32_t), cmp_u32);
    uint64_t k = 0;
    for (uint64_t j = 0; j < d; j++)
      if (k == 0 || a[j] != a[k - 1]) a[k++] = a[j];
    deg[v] = k;
  }
  acc = 0;
  for (uint64_t v = 0; v < nv; v++) { off[v] = acc; acc += deg[v]; }
  off[nv] = acc;
  uint32_t *adj = (uint32_t *)malloc((acc + 1) * sizeof(uint32_t));
  if (!adj) { free(deg); free(pos); free(tmp); return -1; }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)nv; v++)
    memcpy(adj + off[v], tmp + pos[v], deg[v] * sizeof(uint32_t));
  free(tmp);
  free(pos);
  free(deg);
  *adj_out = adj;
  *ne_out = acc;
  return 0;
}

int thvo_generate(uint32_t scale, uint32_t edge_factor, uint64_t seed,
                  double a, double b, double c, int symmetric, uint64_t *off,
                  uint32_t **adj, uint64_t *ne) {
  if (scale == 0 || scale > 32) return -1;
  const uint64_t nv = 1ull << scale;
  const uint64_t n_raw = (uint64_t)edge_factor * nv;
  uint32_t thr[3];
  thvo_rmat_thresholds(a, b, c, thr);
  uint32_t *s = (uint32_t *)malloc((n_raw + 1) * sizeof(uint32_t));
  uint32_t *d = (uint32_t *)malloc((n_raw + 1) * sizeof(uint32_t));
  if (!s || !d) { free(s); free(d); return -1; }
  thvo_rmat_edges(scale, seed, thr, 0, n_raw, s, d);
  const int rc = thvo_build_csr(nv, n_raw, s, d, symmetric, off, adj, ne);
  free(s);
  free(d);
  return rc;
}

void thvo_weights(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  uint64_t seed, uint32_t *w) {
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t u = 0; u < (int64_t)nv; u++)
    for (uint64_t i = off[u]; i < off[u + 1]; i++)
      w[i] = thvo_weight(seed, (uint32_t)u, adj[i]);
}

void thvo_transpose(uint64_t nv, uint64_t ne, const uint64_t *off,
                    const uint32_t *adj, uint64_t *in_off, uint32_t *in_adj,
                    uint32_t *outdeg) {
  uint64_t *cnt = (uint64_t *)calloc(nv + 1, sizeof(uint64_t));
  for (uint64_t u = 0; u < nv; u++) {
    outdeg[u] = (uint32_t)(off[u + 1] - off[u]);
    for (uint64_t i = off[u]; i < off[u + 1]; i++) cnt[adj[i]]++;
  }
  uint64_t acc = 0;
  for (uint64_t v = 0; v < nv; v++) { in_off[v] = acc; acc += cnt[v]; }
  in_off[nv] = acc;
  (void)ne;
  memcpy(cnt, in_off, (nv + 1) * sizeof(uint64_t));
  /* sources visited in increasing order => each in-list sorted by src */
  for (uint64_t u = 0; u < nv; u++)
    for (uint64_t i = off[u]; i < off[u + 1]; i++)
      in_adj[cnt[adj[i]]++] = (uint32_t)u;
  free(cnt);
}

int thvo_sources(uint64_t nv, const uint64_t *off, uint64_t seed, uint32_t n,
                 uint32_t *out) {
  const uint64_t key = thvo_mix64(seed ^ THVO_SOURCE_SALT);
  for (uint32_t j = 0; j < n; j++) {
    int found = 0;
    for (uint64_t t = 0; t < (1ull << 24); t++) {
      const uint64_t cand =
          thvo_mix64(key ^ (((uint64_t)j << 24) | t)) % nv;
      if (off[cand + 1] > off[cand]) { out[j] = (uint32_t)cand; found = 1; break; }
    }
    if (!found) return -1;
  }
  return 0;
}

/* ----------------------------------------------------------- algorithms -- */

static inline uint32_t ld_u32(const uint32_t *p) {
  return __atomic_load_n(p, __ATOMIC_RELAXED);
}

/* atomic min on u32; returns 1 if this call lowered the value */
static inline int atomic_min_u32(uint32_t *p, uint32_t v) {
  uint32_t cur = ld_u32(p);
  while (v < cur) {
    if (__atomic_compare_exchange_n(p, &cur, v, 1, __ATOMIC_RELAXED,
                                    __ATOMIC_RELAXED))
      return 1;
  }
  return 0;
}

int thvo_bfs(uint64_t nv, const uint64_t *off, const uint32_t *adj,
             uint32_t stride, uint32_t src, uint32_t *level) {
  if (src >= nv) return -1;
  const uint32_t inf = (uint32_t)(nv + 1);
  for (uint64_t v = 0; v < nv; v++) level[v] = inf;
  uint32_t *q = (uint32_t *)malloc(nv * sizeof(uint32_t));
  if (!q) return -1;
  uint64_t head = 0, tail = 0;
  level[src] = 1;
  q[tail++] = src;
  while (head < tail) {
    const uint32_t u = q[head++];
    for (uint64_t i = off[u]; i < off[u + 1]; i++) {
      const uint32_t w = adj[i * stride];
      if (level[w] == inf) { level[w] = level[u] + 1; q[tail++] = w; }
    }
  }
  free(q);
  return 0;
}

int thvo_bfs_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                 uint32_t stride, uint32_t src, uint32_t *level) {
  if (src >= nv) return -1;
  const uint32_t inf = (uint32_t)(nv + 1);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)nv; v++) level[v] = inf;
  uint32_t *cur = (uint32_t *)malloc(nv * sizeof(uint32_t));
  uint32_t *nxt = (uint32_t *)malloc(nv * sizeof(uint32_t));
  if (!cur || !nxt) { free(cur); free(nxt); return -1; }
  uint64_t ncur = 1, nnxt;
  cur[0] = src;
  level[src] = 1;
  uint32_t lvl = 1;
  while (ncur) {
    nnxt = 0;
#pragma omp parallel
    {
      uint32_t buf[256];
      int nb = 0;
#pragma omp for schedule(dynamic, 64)
      for (int64_t k = 0; k < (int64_t)ncur; k++) {
        const uint32_t u = cur[k];
        for (uint64_t i = off[u]; i < off[u + 1]; i++) {
          const uint32_t w = adj[i * stride];
          uint32_t expect = inf;
          if (ld_u32(&level[w]) == inf &&
              __atomic_compare_exchange_n(&level[w], &expect, lvl + 1, 0,
                                          __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
            buf[nb++] = w;
            if (nb == 256) {
              uint64_t p = __atomic_fetch_add(&nnxt, 256, __ATOMIC_RELAXED);
              memcpy(nxt + p, buf, sizeof(buf));
              nb = 0;
            }
          }
        }
      }
      if (nb) {
        uint64_t p = __atomic_fetch_add(&nnxt, (uint64_t)nb, __ATOMIC_RELAXED);
        memcpy(nxt + p, buf, (size_t)nb * sizeof(uint32_t));
      }
    }
    uint32_t *t = cur; cur = nxt; nxt = t;
    ncur = nnxt;
    lvl++;
  }
  free(cur);
  free(nxt);
  return 0;
}

int thvo_cc(uint64_t nv, const uint64_t *off, const uint32_t *adj,
            uint32_t stride, uint32_t *label) {
  /* FIFO worklist; the fixed point label[v] = min{u : u reaches v} is unique */
  uint32_t *q = (uint32_t *)malloc((nv + 1) * sizeof(uint32_t));
  unsigned char *inq = (unsigned char *)malloc(nv + 1);
  if (!q || !inq) { free(q); free(inq); return -1; }
  for (uint64_t v = 0; v < nv; v++) { label[v] = (uint32_t)v; q[v] = (uint32_t)v; inq[v] = 1; }
  uint64_t head = 0, count = nv; /* circular buffer of capacity nv */
  while (count) {
    const uint32_t u = q[head];
    head = head + 1 == nv ? 0 : head + 1;
    count--;
    inq[u] = 0;
    const uint32_t lu = label[u];
    for (uint64_t i = off[u]; i < off[u + 1]; i++) {
      const uint32_t w = adj[i * stride];
      if (lu < label[w]) {
        label[w] = lu;
        if (!inq[w]) {
          uint64_t t = head + count;
          if (t >= nv) t -= nv;
          q[t] = w;
          count++;
          inq[w] = 1;
        }
      }
    }
  }
  free(q);
  free(inq);
  return 0;
}

int thvo_cc_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                uint32_t stride, uint32_t *label) {
  unsigned char *act = (unsigned char *)malloc(nv + 1);
  unsigned char *nxt = (unsigned char *)malloc(nv + 1);
  if (!act || !nxt) { free(act); free(nxt); return -1; }
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)nv; v++) { label[v] = (uint32_t)v; act[v] = 1; nxt[v] = 0; }
  int any = 1;
  while (any) {
    any = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : any)
    for (int64_t u = 0; u < (int64_t)nv; u++) {
      if (!act[u]) continue;
      act[u] = 0;
      const uint32_t lu = ld_u32(&label[u]);
      for (uint64_t i = off[u]; i < off[u + 1]; i++) {
        const uint32_t w = adj[i * stride];
        if (lu < ld_u32(&label[w]) && atomic_min_u32(&label[w], lu)) {
          __atomic_store_n(&nxt[w], 1, __ATOMIC_RELAXED);
          any = 1;
        }
      }
    }
    unsigned char *t = act; act = nxt; nxt = t;
  }
  free(act);
  free(nxt);
  return 0;
}

/* edge (dst, weight) accessor for interleaved (w == NULL, stride 2) or split
 * (w != NULL, stride 1) layouts */
static inline void edge_at(const uint32_t *adj, const uint32_t *w,
                           uint32_t stride, uint64_t i, uint32_t *d,
                           uint32_t *wt) {
  if (w) { *d = adj[i]; *wt = w[i]; }
  else { *d = adj[i * stride]; *wt = stride == 2 ? adj[i * 2 + 1] : 1u; }
}

typedef struct { uint64_t key; uint32_t v; } heap_item;

static void heap_push(heap_item *h, uint64_t *n, heap_item it) {
  uint64_t i = (*n)++;
  while (i > 0) {
    uint64_t p = (i - 1) / 2;
    if (h[p].key <= it.key) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = it;
}

static heap_item heap_pop(heap_item *h, uint64_t *n) {
  heap_item top = h[0], last = h[--(*n)];
  uint64_t i = 0;
  for (;;) {
    uint64_t l = 2 * i + 1, r = l + 1, m = i;
    uint64_t mk = last.key;
    if (l < *n && h[l].key < mk) { m = l; mk = h[l].key; }
    if (r < *n && h[r].key < mk) { m = r; }
    if (m == i) break;
    h[i] = h[m];
    i = m;
  }
  if (*n) h[i] = last;
  return top;
}

int thvo_sssp(uint64_t nv, const uint64_t *off, const uint32_t *adj,
              const uint32_t *w, uint32_t stride, uint32_t src,
              uint32_t *dist) {
  if (src >= nv) return -1;
  const uint64_t inf = nv + 1;
  uint64_t *d = (uint64_t *)malloc(nv * sizeof(uint64_t));
  const uint64_t ne = off[nv];
  heap_item *h = (heap_item *)malloc((ne + 2) * sizeof(heap_item));
  if (!d || !h) { free(d); free(h); return -1; }
  for (uint64_t v = 0; v < nv; v++) d[v] = UINT64_MAX;
  uint64_t n = 0;
  d[src] = 1; /* reference encoding: the source holds 1 */
  heap_push(h, &n, (heap_item){1, src});
  while (n) {
    heap_item it = heap_pop(h, &n);
    if (it.key != d[it.v]) continue;
    for (uint64_t i = off[it.v]; i < off[it.v + 1]; i++) {
      uint32_t x, wt;
      edge_at(adj, w, stride, i, &x, &wt);
      const uint64_t nd = it.key + wt;
      if (nd < d[x]) { d[x] = nd; heap_push(h, &n, (heap_item){nd, x}); }
    }
  }
  /* values >= n+1 are never stored by the reference's relaxation */
  for (uint64_t v = 0; v < nv; v++) dist[v] = (uint32_t)(d[v] < inf ? d[v] : inf);
  free(d);
  free(h);
  return 0;
}

int thvo_sssp_par(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  const uint32_t *w, uint32_t stride, uint32_t src,
                  uint32_t *dist) {
  if (src >= nv) return -1;
  const uint32_t inf = (uint32_t)(nv + 1);
  unsigned char *act = (unsigned char *)calloc(nv + 1, 1);
  unsigned char *nxt = (unsigned char *)calloc(nv + 1, 1);
  if (!act || !nxt) { free(act); free(nxt); return -1; }
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)nv; v++) dist[v] = inf;
  dist[src] = 1;
  act[src] = 1;
  int any = 1;
  while (any) {
    any = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : any)
    for (int64_t u = 0; u < (int64_t)nv; u++) {
      if (!act[u]) continue;
      act[u] = 0;
      const uint64_t du = ld_u32(&dist[u]);
      for (uint64_t i = off[u]; i < off[u + 1]; i++) {
        uint32_t x, wt;
        edge_at(adj, w, stride, i, &x, &wt);
        const uint64_t nd = du + wt;
        if (nd < ld_u32(&dist[x]) && atomic_min_u32(&dist[x], (uint32_t)nd)) {
          __atomic_store_n(&nxt[x], 1, __ATOMIC_RELAXED);
          any = 1;
        }
      }
    }
    unsigned char *t = act; act = nxt; nxt = t;
  }
  free(act);
  free(nxt);
  return 0;
}

int thvo_pagerank_csc(uint64_t nv, const uint64_t *in_off,
                      const uint32_t *in_adj, const uint32_t *outdeg,
                      uint32_t iters, double damping, double *rank) {
  double *contrib = (double *)malloc(nv * sizeof(double));
  if (!contrib) return -1;
  const double n = (double)nv;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)nv; v++) rank[v] = 1.0 / n;
  for (uint32_t it = 0; it < iters; it++) {
    double dangling = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : dangling)
    for (int64_t u = 0; u < (int64_t)nv; u++) {
      if (outdeg[u]) contrib[u] = rank[u] / (double)outdeg[u];
      else { contrib[u] = 0.0; dangling += rank[u]; }
    }
    const double base = (1.0 - damping) / n + damping * dangling / n;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < (int64_t)nv; v++) {
      double s = 0.0;
      for (uint64_t i = in_off[v]; i < in_off[v + 1]; i++) s += contrib[in_adj[i]];
      rank[v] = base + damping * s;
    }
  }
  free(contrib);
  return 0;
}

int thvo_pagerank(uint64_t nv, const uint64_t *off, const uint32_t *adj,
                  uint32_t stride, uint32_t iters, double damping,
                  double *rank) {
  const uint64_t ne = off[nv];
  uint32_t *plain = NULL;
  const uint32_t *a = adj;
  if (stride != 1) {
    plain = (uint32_t *)malloc((ne + 1) * sizeof(uint32_t));
    if (!plain) return -1;
    for (uint64_t i = 0; i < ne; i++) plain[i] = adj[i * stride];
    a = plain;
  }
  uint64_t *in_off = (uint64_t *)malloc((nv + 1) * sizeof(uint64_t));
  uint32_t *in_adj = (uint32_t *)malloc((ne + 1) * sizeof(uint32_t));
  uint32_t *outdeg = (uint32_t *)malloc((nv + 1) * sizeof(uint32_t));
  int rc = -1;
  if (in_off && in_adj && outdeg) {
    thvo_transpose(nv, ne, off, a, in_off, in_adj, outdeg);
    rc = thvo_pagerank_csc(nv, in_off, in_adj, outdeg, iters, damping, rank);
  }
  free(in_off);
  free(in_adj);
  free(outdeg);
  free(plain);
  return rc;
}

/* The reference's PageRank constants are floats (src/common.cuh:48-49,
 * TOLERANCE 0.001f, ALPHA 0.85f); its expressions mix them with doubles, and
 * the same C expressions below give the same promoted values. */
static const float kRefAlpha = 0.85f, kRefTol = 0.001f;

/* Pull: r0 = 1/N (src/graph.cuh:239-240); every round, each active vertex
 * sums r(u)/outdeg(u) over its in-edges with the values of the previous
 * round (the gather kernels, src/pr/pr_kernels.cu:23-55 and their demand /
 * filter forms, all run before the update), then r = (1-a) + a*sum and the
 * vertex stays active while |change| > tol (PR32_Update_Values,
 * pr_kernels.cu:449-476); an inactive vertex never returns.  Rounds run while
 * any vertex is active (src/pr/pr.cu:49-500). */
int thvo_pagerank_ref_pull(uint64_t nv, const uint64_t *in_off,
                           const uint32_t *in_adj, const uint32_t *outdeg,
                           uint32_t max_rounds, double *rank, uint32_t *rounds) {
  double *sum = (double *)malloc((nv + 1) * sizeof(double));
  unsigned char *act = (unsigned char *)malloc(nv + 1);
  if (!sum || !act) { free(sum); free(act); return -1; }
  for (uint64_t v = 0; v < nv; v++) { rank[v] = 1.0 / (double)nv; act[v] = 1; }
  uint64_t nact = nv;
  uint32_t r = 0;
  while (nact) {
    if (r == max_rounds) { free(sum); free(act); *rounds = r; return -2; }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)nv; v++) {
      if (!act[v]) continue;
      double s = 0.0;
      for (uint64_t i = in_off[v]; i < in_off[v + 1]; i++) {
        const uint32_t u = in_adj[i];
        if (outdeg[u]) s += rank[u] / (double)outdeg[u];
      }
      sum[v] = s;
    }
    nact = 0;
#pragma omp parallel for schedule(static) reduction(+ : nact)
    for (int64_t v = 0; v < (int64_t)nv; v++) {
      if (!act[v]) continue;
      const double t = (1 - kRefAlpha) + kRefAlpha * sum[v];
      const double diff = t > rank[v] ? t - rank[v] : rank[v] - t;
      rank[v] = t;
      act[v] = diff > kRefTol;
      nact += act[v];
    }
    r++;
  }
  free(sum);
  free(act);
  *rounds = r;
  return 0;
}

/* Push, residual form: r0 = 1-a, delta0 = (1-a)*a/outdeg computed in float,
 * residual 0, every vertex active (src/graph.cuh:233-237).  Every round
 * clears the frontier (src/pr/pr.cu:1067-1077), each active u adds delta(u)
 * to residual(w) over its out-edges (PR32_Static_Kernel_PUSH and its demand /
 * filter forms, pr_kernels.cu:504-681), then every vertex whose residual
 * exceeds tol takes it: r += residual, delta = residual*a/outdeg,
 * residual = 0, active (PR32_Update_Values_PUSH, pr_kernels.cu:846-860).
 * Residuals at or under tol stay and keep accumulating. */
int thvo_pagerank_ref_push(uint64_t nv, const uint64_t *off,
                           const uint32_t *adj, uint32_t stride,
                           uint32_t max_rounds, double *rank, uint32_t *rounds) {
  double *delta = (double *)malloc((nv + 1) * sizeof(double));
  double *res = (double *)malloc((nv + 1) * sizeof(double));
  unsigned char *act = (unsigned char *)malloc(nv + 1);
  if (!delta || !res || !act) { free(delta); free(res); free(act); return -1; }
  for (uint64_t v = 0; v < nv; v++) {
    rank[v] = (double)(1.0f - kRefAlpha);
    delta[v] = (double)((1.0f - kRefAlpha) * kRefAlpha / (float)(off[v + 1] - off[v]));
    res[v] = 0.0;
    act[v] = 1;
  }
  uint64_t nact = nv;
  uint32_t r = 0;
  while (nact) {
    if (r == max_rounds) { free(delta); free(res); free(act); *rounds = r; return -2; }
    for (uint64_t u = 0; u < nv; u++) {
      if (!act[u]) continue;
      for (uint64_t i = off[u]; i < off[u + 1]; i++) res[adj[i * stride]] += delta[u];
    }
    nact = 0;
    for (uint64_t v = 0; v < nv; v++) {
      if (res[v] > kRefTol) {
        rank[v] += res[v];
        delta[v] = res[v] * kRefAlpha / (double)(off[v + 1] - off[v]);
        res[v] = 0.0;
        act[v] = 1;
        nact++;
      } else {
        act[v] = 0;
      }
    }
    r++;
  }
  free(delta);
  free(res);
  free(act);
  *rounds = r;
  return 0;
}

uint64_t thvo_reached_edges(uint64_t nv, const uint64_t *off,
                            const uint32_t *val) {
  uint64_t s = 0;
  const uint32_t inf = (uint32_t)(nv + 1);
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t v = 0; v < (int64_t)nv; v++)
    if (val[v] < inf) s += off[v + 1] - off[v];
  return s;
}

/* ---------------------------------------------------------------- files -- */

static int write_all(FILE *f, const void *p, size_t n) {
  return fwrite(p, 1, n, f) == n ? 0 : -1;
}

int thvo_write_csr(const char *path, uint64_t nv, uint64_t ne,
                   const uint64_t *off, const uint32_t *adj,
                   const uint32_t *w) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  int rc = write_all(f, &nv, 8) | write_all(f, &ne, 8) |
           write_all(f, off, nv * 8) | write_all(f, adj, ne * 4);
  if (w) rc |= write_all(f, w, ne * 4);
  else {
    const uint32_t twenty = 20; /* converter default weight */
    for (uint64_t i = 0; i < ne && !rc; i++) rc |= write_all(f, &twenty, 4);
  }
  return fclose(f) | rc;
}

int thvo_write_csc(const char *path, uint64_t nv, uint64_t ne,
                   const uint64_t *in_off, const uint32_t *in_adj,
                   const uint32_t *outdeg) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  int rc = write_all(f, &nv, 8) | write_all(f, &ne, 8) |
           write_all(f, in_off, nv * 8) | write_all(f, in_adj, ne * 4) |
           write_all(f, outdeg, nv * 4);
  return fclose(f) | rc;
}

int thvo_write_wcsr(const char *path, uint64_t nv, uint64_t ne,
                    const uint64_t *off, const uint32_t *adj,
                    const uint32_t *w) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  int rc = write_all(f, &nv, 8) | write_all(f, &ne, 8) |
           write_all(f, off, nv * 8);
  uint32_t buf[2048];
  for (uint64_t i = 0; i < ne && !rc;) {
    uint64_t k = 0;
    for (; k < 1024 && i < ne; k++, i++) {
      buf[2 * k] = adj[i];
      buf[2 * k + 1] = w ? w[i] : 20u;
    }
    rc |= write_all(f, buf, k * 8);
  }
  return fclose(f) | rc;
}

int thvo_write_values(const char *path, const void *vals, uint64_t n,
                      uint32_t elem_size) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  int rc = write_all(f, vals, n * elem_size);
  return fclose(f) | rc;
}

double thvo_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int thvo_threads(void) { return omp_get_max_threads(); }
void thvo_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
