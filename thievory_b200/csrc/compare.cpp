// compare -- checks two results/values.bin files, the drop-in for the
// reference's comparer/compare.cpp (same flags: --input1 --input2 --type
// --vertices).  Integers must match exactly; doubles within an absolute
// tolerance (1e-3 as in compare.cpp:155, or --tolerance).
//
// Differences from the reference tool, all deliberate fixes:
// - u32 files are read as 4-byte values (compare.cpp:59-60 reads nV * 8
//   bytes into a u32 array);
// - vertex indices are 64-bit (compare.cpp:74 counts in u32);
// - a file shorter than the vertex count is an error, not a silent
//   comparison against zero-filled values;
// - the exit status is 0 only when the files match (the reference always
//   exits 0), and a summary line gives the mismatch count;
// - NaN never matches.
#include <cerrno>
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

enum Kind { kU32 = 0, kU64 = 1, kDouble = 2 };

void usage(const char *prog) {
  fprintf(stderr,
          "Usage: %s --input1 <values.bin> --input2 <values.bin> --vertices <n>\n"
          "          [--type 0|1|2] [--tolerance <abs>] [--max-report <k>]\n"
          "  --type       0 = u32 (BFS/CC/SSSP, default), 1 = u64, 2 = double (PageRank)\n"
          "  --tolerance  absolute tolerance for doubles (default 1e-3)\n"
          "  --max-report mismatches printed before the summary (default 20)\n",
          prog);
}

template <typename T>
bool read_values(const char *path, uint64_t n, std::vector<T> &out) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "Error: cannot open %s: %s\n", path, strerror(errno));
    return false;
  }
  out.resize(n);
  const size_t got = n ? fread(out.data(), sizeof(T), n, f) : 0;
  fclose(f);
  if (got != n) {
    fprintf(stderr, "Error: %s holds %zu values, expected %" PRIu64 "\n", path, got, n);
    return false;
  }
  return true;
}

void print_value(uint32_t v) { printf("%" PRIu32, v); }
void print_value(uint64_t v) { printf("%" PRIu64, v); }
void print_value(double v) { printf("%.17g", v); }

bool equal(uint32_t a, uint32_t b, double) { return a == b; }
bool equal(uint64_t a, uint64_t b, double) { return a == b; }
bool equal(double a, double b, double tol) { return std::fabs(a - b) <= tol; }  // NaN: false

template <typename T>
int compare(const char *p1, const char *p2, uint64_t n, double tol, uint64_t max_report) {
  std::vector<T> a, b;
  if (!read_values(p1, n, a) || !read_values(p2, n, b)) return 2;
  uint64_t bad = 0;
  for (uint64_t i = 0; i < n; i++) {
    if (equal(a[i], b[i], tol)) continue;
    if (bad < max_report) {
      printf("Arrays do not match at: %" PRIu64 "\n", i);
      print_value(a[i]);
      printf(" | ");
      print_value(b[i]);
      printf("\n");
    }
    bad++;
  }
  printf("Mismatches: %" PRIu64 " of %" PRIu64 "\n", bad, n);
  return bad ? 1 : 0;
}

}  // namespace

int main(int argc, char **argv) {
  const char *in1 = nullptr, *in2 = nullptr;
  uint64_t n = 0, max_report = 20;
  int kind = kU32;
  double tol = 1e-3;
  bool have_n = false;
  for (int i = 1; i < argc; i++) {
    const char *k = argv[i];
    if (i + 1 >= argc) {
      usage(argv[0]);
      return 2;
    }
    const char *v = argv[++i];
    char *end = nullptr;
    errno = 0;
    if (!strcmp(k, "--input1")) {
      in1 = v;
    } else if (!strcmp(k, "--input2")) {
      in2 = v;
    } else if (!strcmp(k, "--vertices")) {
      n = strtoull(v, &end, 10);
      have_n = true;
    } else if (!strcmp(k, "--type")) {
      kind = (int)strtol(v, &end, 10);
    } else if (!strcmp(k, "--tolerance")) {
      tol = strtod(v, &end);
    } else if (!strcmp(k, "--max-report")) {
      max_report = strtoull(v, &end, 10);
    } else {
      fprintf(stderr, "Error: unknown option %s\n", k);
      usage(argv[0]);
      return 2;
    }
    if (end && (*end || errno)) {
      fprintf(stderr, "Error: bad value for %s: %s\n", k, v);
      return 2;
    }
  }
  if (!in1 || !in2 || !have_n || kind < kU32 || kind > kDouble || !(tol >= 0)) {
    usage(argv[0]);
    return 2;
  }
  printf("Comparing %s, %" PRIu64 " vertices\n",
         kind == kU32 ? "UINT32" : kind == kU64 ? "UINT64" : "DOUBLES", n);
  if (kind == kU32) return compare<uint32_t>(in1, in2, n, tol, max_report);
  if (kind == kU64) return compare<uint64_t>(in1, in2, n, tol, max_report);
  return compare<double>(in1, in2, n, tol, max_report);
}
