// Text edge list -> the converter's byte formats, sorting on the GPU.
//
// Replaces converter/converter.cpp's ConvertTxtToBCSR (.csr, and .wcsr with
// its "liberator" {dst, w} pairs, :676-808) and ConvertTxtToBCSC (.csc,
// :483-589) with the same output bytes:
// - the first `skip` lines are dropped (converter default 4, :815);
// - each later line is read as `src dst [w]` with istream semantics: a
//   field that fails to parse keeps the value of the previous line, and
//   once one field fails the rest of the line is not read (the converter
//   reuses src/dest/weight across lines, :693-708); w is read only for
//   weighted inputs (-DWEIGHTED, :706), else 20 (:693);
// - undirected inputs add dst -> src (-DUNDIRECTED, :711);
// - duplicates and self-loops are kept, nv = max id + 1 (:718-722);
// - edges sorted by (src, dst), by (dst, src) for CSC.
// The sort is a stable radix sort, so duplicate pairs keep their input order
// (the converter's std::sort leaves the weight order of duplicate pairs
// unspecified; identical for unweighted inputs).
#include <cub/cub.cuh>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "thv_internal.h"

namespace thv {

namespace {

struct FileCloser {
  void operator()(FILE *f) const {
    if (f) fclose(f);
  }
};

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// istream >> unsigned long long on one line: skip blanks, optional '+',
// digits.  Returns false (field not read) on no digits, a '-' sign or
// overflow.
bool read_u64(const char *&p, const char *end, uint64_t *out) {
  while (p < end && is_space(*p)) p++;
  if (p < end && *p == '+') p++;
  if (p >= end || *p < '0' || *p > '9') return false;
  uint64_t v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    const uint64_t d = (uint64_t)(*p - '0');
    if (v > (UINT64_MAX - d) / 10) return false;
    v = v * 10 + d;
    p++;
  }
  *out = v;
  return true;
}

__global__ void cv_offsets(const unsigned long long *keys, uint64_t ne, uint64_t nv,
                           uint64_t *off) {
  // off[x] = first sorted edge whose key vertex is >= x, x in [0, nv]
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t u = keys[i] >> 32;
    const uint64_t prev = i == 0 ? 0 : (keys[i - 1] >> 32) + 1;
    for (uint64_t x = prev; x <= u; x++) off[x] = i;
    if (i == ne - 1)
      for (uint64_t x = u + 1; x <= nv; x++) off[x] = ne;
  }
}

__global__ void cv_low_words(const unsigned long long *keys, uint64_t ne, uint32_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)keys[i];
}

template <typename T>
struct DevBuf {
  T *p = nullptr;
  ~DevBuf() { dev_free(p); }
};

}  // namespace

thv_status convert_edge_list(const char *txt, const char *out_path, thv_format fmt,
                             uint32_t skip, uint32_t flags, int device, uint64_t *nv_out,
                             uint64_t *ne_out) {
  if (!txt || !out_path) return fail(THV_EINVAL, "null path");
  if (fmt != THV_FMT_CSR && fmt != THV_FMT_CSC && fmt != THV_FMT_WCSR)
    return fail(THV_EINVAL, "unknown output format %d", (int)fmt);
  const bool weighted = flags & THV_CONVERT_WEIGHTED;
  const bool undirected = flags & THV_CONVERT_UNDIRECTED;
  // ---------------------------------------------------------------- parse
  std::unique_ptr<FILE, FileCloser> f(fopen(txt, "rb"));
  if (!f) return fail(THV_EIO, "cannot open %s: %s", txt, strerror(errno));
  std::vector<char> buf;
  {
    char chunk[1 << 16];
    size_t n;
    while ((n = fread(chunk, 1, sizeof(chunk), f.get())) > 0) buf.insert(buf.end(), chunk, chunk + n);
    if (ferror(f.get())) return fail(THV_EIO, "read error on %s", txt);
  }
  std::vector<unsigned long long> keys;  // (key vertex << 32) | other vertex
  std::vector<uint32_t> wts;
  std::vector<uint32_t> outdeg;  // CSC: out-degree per vertex
  uint64_t src = 0, dst = 0, w = 20, maxid = 0;
  bool any = false;
  const char *p = buf.data(), *end = buf.data() + buf.size();
  uint64_t line = 0;
  while (p < end) {
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    const char *le = nl ? nl : end;
    if (line++ >= skip) {
      const char *q = p;
      if (read_u64(q, le, &src) && read_u64(q, le, &dst) && weighted) read_u64(q, le, &w);
      if (src > 0xFFFFFFFEull || dst > 0xFFFFFFFEull)
        return fail(THV_EUNSUPPORTED, "%s:%llu: vertex id above 2^32 - 2", txt,
                    (unsigned long long)line);
      const uint32_t wv = (uint32_t)w;
      auto add = [&](uint64_t a, uint64_t b) {
        keys.push_back(fmt == THV_FMT_CSC ? (b << 32) | a : (a << 32) | b);
        if (fmt != THV_FMT_CSC) wts.push_back(wv);
      };
      add(src, dst);
      if (undirected) add(dst, src);
      maxid = std::max(maxid, std::max(src, dst));
      any = true;
    }
    p = nl ? nl + 1 : end;
  }
  const uint64_t nv = any ? maxid + 1 : 1;  // the converter counts vertex 0 always
  const uint64_t ne = keys.size();
  if (fmt == THV_FMT_CSC) {
    outdeg.assign(nv, 0);
    for (unsigned long long k : keys) outdeg[k & 0xFFFFFFFFull]++;
  }
  // ------------------------------------------------------------ GPU sort
  THV_CUDA(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  THV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};
  std::vector<uint64_t> off(nv + 1, 0);
  std::vector<uint32_t> other(ne), sorted_w;
  if (ne) {
    DevBuf<unsigned long long> k0, k1;
    DevBuf<uint32_t> v0, v1, lo;
    DevBuf<uint64_t> d_off;
    DevBuf<char> tmp;
    THV_TRY(dev_alloc((void **)&k0.p, ne * 8, "convert keys"));
    THV_TRY(dev_alloc((void **)&k1.p, ne * 8, "convert keys"));
    THV_TRY(dev_alloc((void **)&d_off.p, (nv + 1) * 8, "convert offsets"));
    THV_TRY(dev_alloc((void **)&lo.p, ne * 4, "convert ids"));
    const bool with_w = fmt != THV_FMT_CSC;
    if (with_w) {
      THV_TRY(dev_alloc((void **)&v0.p, ne * 4, "convert weights"));
      THV_TRY(dev_alloc((void **)&v1.p, ne * 4, "convert weights"));
      THV_CUDA(cudaMemcpyAsync(v0.p, wts.data(), ne * 4, cudaMemcpyHostToDevice, st));
    }
    THV_CUDA(cudaMemcpyAsync(k0.p, keys.data(), ne * 8, cudaMemcpyHostToDevice, st));
    cub::DoubleBuffer<unsigned long long> kb(k0.p, k1.p);
    cub::DoubleBuffer<uint32_t> vb(v0.p, v1.p);
    size_t tb = 0;
    if (with_w)
      THV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, (int64_t)ne, 0, 64, st));
    else
      THV_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, kb, (int64_t)ne, 0, 64, st));
    THV_TRY(dev_alloc((void **)&tmp.p, tb + 16, "convert sort scratch"));
    if (with_w)
      THV_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kb, vb, (int64_t)ne, 0, 64, st));
    else
      THV_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, kb, (int64_t)ne, 0, 64, st));
    const int grid = 1024;
    cv_offsets<<<grid, 256, 0, st>>>(kb.Current(), ne, nv, d_off.p);
    cv_low_words<<<grid, 256, 0, st>>>(kb.Current(), ne, lo.p);
    THV_CUDA(cudaGetLastError());
    THV_CUDA(cudaMemcpyAsync(off.data(), d_off.p, (nv + 1) * 8, cudaMemcpyDeviceToHost, st));
    THV_CUDA(cudaMemcpyAsync(other.data(), lo.p, ne * 4, cudaMemcpyDeviceToHost, st));
    if (with_w) {
      sorted_w.resize(ne);
      THV_CUDA(cudaMemcpyAsync(sorted_w.data(), vb.Current(), ne * 4, cudaMemcpyDeviceToHost, st));
    }
    THV_CUDA(cudaStreamSynchronize(st));
  }
  // ---------------------------------------------------------------- write
  std::unique_ptr<FILE, FileCloser> o(fopen(out_path, "wb"));
  if (!o) return fail(THV_EIO, "cannot create %s: %s", out_path, strerror(errno));
  bool ok = fwrite(&nv, 8, 1, o.get()) == 1 && fwrite(&ne, 8, 1, o.get()) == 1;
  ok = ok && fwrite(off.data(), 8, nv, o.get()) == nv;  // no trailing entry
  if (fmt == THV_FMT_WCSR) {
    std::vector<uint32_t> pairs;
    pairs.reserve(std::min<uint64_t>(2 * ne, 1u << 21));
    for (uint64_t i = 0; ok && i < ne; i++) {
      pairs.push_back(other[i]);
      pairs.push_back(sorted_w[i]);
      if (pairs.size() >= (1u << 21) || i + 1 == ne) {
        ok = fwrite(pairs.data(), 4, pairs.size(), o.get()) == pairs.size();
        pairs.clear();
      }
    }
  } else {
    ok = ok && (ne == 0 || fwrite(other.data(), 4, ne, o.get()) == ne);
    if (fmt == THV_FMT_CSR) ok = ok && (ne == 0 || fwrite(sorted_w.data(), 4, ne, o.get()) == ne);
    else ok = ok && fwrite(outdeg.data(), 4, nv, o.get()) == nv;
  }
  if (!ok) return fail(THV_EIO, "write to %s failed", out_path);
  if (nv_out) *nv_out = nv;
  if (ne_out) *ne_out = ne;
  return THV_OK;
}

}  // namespace thv
