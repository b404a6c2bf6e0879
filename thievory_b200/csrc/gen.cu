// Seeded RMAT generator on the GPU (graph ingest; not on the traversal path).
//
// The definition is the oracle's (oracle/thv_oracle.c): edge i draws
// ceil(scale/2) splitmix64 words keyed by (seed, i); each 32-bit half picks a
// quadrant against floor(p * 2^32) thresholds; ids go through a seeded
// bijection of [0, 2^scale); self-loops and duplicates are removed and the
// CSR is sorted by (src, dst).  Weights are a hash of (seed, src, dst) in
// [1, 64].  Output bytes are identical to the oracle's for the same inputs.
// Converter layouts written afterwards: converter/converter.cpp:676-805.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "thv_internal.h"

namespace thv {

static constexpr uint64_t kPermSalt = 0x5045524D55544531ull;
static constexpr uint64_t kWeightSalt = 0x5745494748543634ull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct GenParams {
  uint64_t key;       // mix64(seed)
  uint64_t pk[4];     // permutation round keys
  uint64_t wkey;      // weight key
  uint32_t thr[3];
  uint32_t scale;
};

__device__ __forceinline__ uint64_t permute(uint64_t x, const GenParams &p) {
  const uint64_t mask = p.scale >= 64 ? ~0ull : ((1ull << p.scale) - 1);
  const uint32_t h = (p.scale + 1) / 2;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint64_t k = p.pk[r];
    x = (x * (k | 1ull)) & mask;
    x ^= x >> h;
    x = (x + (k >> 17)) & mask;
  }
  return x;
}

__global__ void gen_keys(GenParams p, uint64_t count, int symmetric,
                         unsigned long long *keys) {
  const uint32_t words = (p.scale + 1) / 2;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u = 0, v = 0;
    for (uint32_t k = 0; k < words; k++) {
      const uint64_t x = mix64(p.key ^ ((i << 5) | k));
#pragma unroll
      for (uint32_t half = 0; half < 2; half++) {
        const uint32_t lvl = 2 * k + half;
        if (lvl < p.scale) {
          const uint32_t r = half ? (uint32_t)(x >> 32) : (uint32_t)x;
          const uint32_t ub = r >= p.thr[1];
          const uint32_t vb = (r >= p.thr[0] && r < p.thr[1]) || r >= p.thr[2];
          u = (u << 1) | ub;
          v = (v << 1) | vb;
        }
      }
    }
    u = permute(u, p);
    v = permute(v, p);
    const bool loop = u == v;
    keys[i] = loop ? ~0ull : ((u << 32) | v);
    if (symmetric) keys[count + i] = loop ? ~0ull : ((v << 32) | u);
  }
}

// off[x] = first edge index with src >= x, for x in [0, nv]; keys sorted.
__global__ void keys_to_offsets(const unsigned long long *keys, uint64_t ne,
                                uint64_t nv, uint64_t *off) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t u = keys[i] >> 32;
    const uint64_t prev = i == 0 ? 0 : (keys[i - 1] >> 32) + 1;
    for (uint64_t x = prev; x <= u; x++) off[x] = i;
    if (i == ne - 1)
      for (uint64_t x = u + 1; x <= nv; x++) off[x] = ne;
  }
}

__global__ void keys_to_edges(const unsigned long long *keys, uint64_t ne,
                              int weighted, uint64_t wkey, uint32_t *edges) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    const uint32_t dst = (uint32_t)k;
    if (weighted) {
      edges[2 * i] = dst;
      edges[2 * i + 1] = 1u + (uint32_t)(mix64(wkey ^ k) & 63u);
    } else {
      edges[i] = dst;
    }
  }
}

__global__ void swap_halves(unsigned long long *keys, uint64_t ne) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    keys[i] = (k << 32) | (k >> 32);
  }
}

__global__ void offsets_to_degree(const uint64_t *off, uint64_t nv, uint32_t *deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
}

// Sort keys in place (d0 holds the input; d1 scratch); returns the buffer
// holding the sorted, de-duplicated keys and its length (sentinel dropped).
static thv_status sort_unique(unsigned long long *&d0, unsigned long long *&d1,
                              uint64_t n, uint32_t end_bit, uint64_t *ne_out) {
  cub::DoubleBuffer<unsigned long long> db(d0, d1);
  size_t tb = 0;
  THV_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)n, 0, (int)end_bit));
  void *tmp = nullptr;
  THV_TRY(dev_alloc(&tmp, tb, "sort scratch"));
  cudaError_t e = cub::DeviceRadixSort::SortKeys(tmp, tb, db, (int64_t)n, 0, (int)end_bit);
  dev_free(tmp);
  if (e != cudaSuccess) return fail(THV_ECUDA, "radix sort: %s", cudaGetErrorString(e));
  unsigned long long *sorted = db.Current(), *other = db.Alternate();
  int64_t *d_cnt = nullptr;
  THV_TRY(dev_alloc((void **)&d_cnt, 8, "unique count"));
  tb = 0;
  THV_CUDA(cub::DeviceSelect::Unique(nullptr, tb, sorted, other, d_cnt, (int64_t)n));
  THV_TRY(dev_alloc(&tmp, tb, "unique scratch"));
  e = cub::DeviceSelect::Unique(tmp, tb, sorted, other, d_cnt, (int64_t)n);
  dev_free(tmp);
  if (e != cudaSuccess) { dev_free(d_cnt); return fail(THV_ECUDA, "unique: %s", cudaGetErrorString(e)); }
  int64_t cnt = 0;
  THV_CUDA(cudaMemcpy(&cnt, d_cnt, 8, cudaMemcpyDeviceToHost));
  dev_free(d_cnt);
  uint64_t ne = (uint64_t)cnt;
  if (ne) {
    unsigned long long last = 0;
    THV_CUDA(cudaMemcpy(&last, other + ne - 1, 8, cudaMemcpyDeviceToHost));
    if (last == ~0ull) ne--;
  }
  d0 = other;  // result
  d1 = sorted;
  *ne_out = ne;
  return THV_OK;
}

thv_status graph_adopt(uint64_t nv, uint64_t ne, thv_format fmt, uint32_t esz,
                       std::vector<uint64_t> &off, const void *d_edges,
                       std::vector<uint32_t> &outdeg, bool symmetric, int device,
                       thv_graph **out);

thv_status generate_rmat(const thv_rmat_opts *o, thv_format fmt, int device,
                         thv_graph **out) {
  if (o->scale == 0 || o->scale > 31)
    return fail(THV_EINVAL, "scale must be in [1, 31]");
  if (o->a < 0 || o->b < 0 || o->c < 0 || o->a + o->b + o->c > 1.0)
    return fail(THV_EINVAL, "bad RMAT probabilities");
  THV_CUDA(cudaSetDevice(device));
  const uint64_t nv = 1ull << o->scale;
  const uint64_t raw = (uint64_t)o->edge_factor * nv;
  const uint64_t n = o->symmetric ? 2 * raw : raw;
  GenParams p{};
  p.key = mix64(o->seed);
  const uint64_t pkey = mix64(o->seed ^ kPermSalt);
  for (int r = 0; r < 4; r++) p.pk[r] = mix64(pkey + (uint64_t)r);
  p.wkey = mix64(o->seed ^ kWeightSalt);
  p.scale = o->scale;
  const double two32 = 4294967296.0;
  const double ca = o->a, cb = o->a + o->b, cc = o->a + o->b + o->c;
  p.thr[0] = ca >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(ca * two32);
  p.thr[1] = cb >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(cb * two32);
  p.thr[2] = cc >= 1.0 ? 0xFFFFFFFFu : (uint32_t)(cc * two32);

  unsigned long long *d0 = nullptr, *d1 = nullptr;
  THV_TRY(dev_alloc((void **)&d0, n * 8 + 16, "generator keys"));
  thv_status s = dev_alloc((void **)&d1, n * 8 + 16, "generator keys");
  if (s != THV_OK) { dev_free(d0); return s; }
  auto cleanup = [&]() { dev_free(d0); dev_free(d1); };
  gen_keys<<<4096, 256>>>(p, raw, o->symmetric ? 1 : 0, d0);
  if (cudaGetLastError() != cudaSuccess) { cleanup(); return fail(THV_ECUDA, "gen_keys launch"); }
  uint64_t ne = 0;
  s = sort_unique(d0, d1, n, 64, &ne);
  if (s != THV_OK) { cleanup(); return s; }
  std::vector<uint64_t> off(nv + 1, 0);
  std::vector<uint32_t> outdeg;
  uint64_t *d_off = nullptr;
  uint32_t *d_edges = nullptr;
  const bool weighted = fmt == THV_FMT_WCSR;
  const uint32_t esz = weighted ? 8 : 4;
  s = dev_alloc((void **)&d_off, (nv + 1) * 8, "generator offsets");
  if (s == THV_OK) s = dev_alloc((void **)&d_edges, ne * esz + 16, "generator edges");
  if (s != THV_OK) { cleanup(); dev_free(d_off); return s; }
  auto cleanup2 = [&]() { cleanup(); dev_free(d_off); dev_free(d_edges); };
  if (fmt == THV_FMT_CSC) {
    // out-degrees from the CSR order, then re-sort by (dst, src)
    if (ne) keys_to_offsets<<<4096, 256>>>(d0, ne, nv, d_off);
    else cudaMemset(d_off, 0, (nv + 1) * 8);
    uint32_t *d_deg = nullptr;
    s = dev_alloc((void **)&d_deg, nv * 4 + 16, "out-degrees");
    if (s != THV_OK) { cleanup2(); return s; }
    offsets_to_degree<<<4096, 256>>>(d_off, nv, d_deg);
    outdeg.resize(nv);
    cudaMemcpy(outdeg.data(), d_deg, nv * 4, cudaMemcpyDeviceToHost);
    dev_free(d_deg);
    swap_halves<<<4096, 256>>>(d0, ne);
    cub::DoubleBuffer<unsigned long long> db(d0, d1);
    size_t tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)ne, 0, 64);
    void *tmp = nullptr;
    s = dev_alloc(&tmp, tb, "sort scratch");
    if (s != THV_OK) { cleanup2(); return s; }
    cub::DeviceRadixSort::SortKeys(tmp, tb, db, (int64_t)ne, 0, 64);
    dev_free(tmp);
    if (db.Current() != d0) std::swap(d0, d1);
  }
  if (ne) keys_to_offsets<<<4096, 256>>>(d0, ne, nv, d_off);
  else cudaMemset(d_off, 0, (nv + 1) * 8);
  keys_to_edges<<<4096, 256>>>(d0, ne, weighted ? 1 : 0, p.wkey, d_edges);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { cleanup2(); return fail(THV_ECUDA, "generator: %s", cudaGetErrorString(e)); }
  e = cudaMemcpy(off.data(), d_off, (nv + 1) * 8, cudaMemcpyDeviceToHost);
  dev_free(d0);
  dev_free(d1);
  d0 = d1 = nullptr;
  dev_free(d_off);
  d_off = nullptr;
  if (e != cudaSuccess) { dev_free(d_edges); return fail(THV_ECUDA, "copy offsets"); }
  const thv_format gfmt = fmt;
  s = graph_adopt(nv, ne, gfmt, esz, off, d_edges, outdeg, o->symmetric != 0, device, out);
  dev_free(d_edges);
  return s;
}

}  // namespace thv
