// convert -- text edge list to .csr / .csc / .wcsr, the drop-in for the
// reference's converter/converter.cpp command line (`--input`, `--type`,
// `--skip`; -DWEIGHTED and -DUNDIRECTED become the runtime flags
// `--weighted` and `--undirected`).  The output name is the input's with
// its extension replaced (g.txt -> g.csr / g.csc / g.wcsr; the reference
// writes "g..wcsr" for WCSR, converter.cpp:777), or `--output`.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "thv.h"

static void usage(const char *prog) {
  fprintf(stderr,
          "Usage: %s --input <edges.txt> [--type csr|csc|wcsr] [--skip <lines>]\n"
          "          [--weighted] [--undirected] [--output <path>] [--device <id>]\n"
          "  --skip  header lines to drop (default 4, as the reference converter)\n",
          prog);
}

int main(int argc, char **argv) {
  std::string input, type = "csr", output;
  unsigned skip = 4, flags = 0;
  int device = 0;
  for (int i = 1; i < argc; i++) {
    const std::string k = argv[i];
    if (k == "--weighted") { flags |= THV_CONVERT_WEIGHTED; continue; }
    if (k == "--undirected") { flags |= THV_CONVERT_UNDIRECTED; continue; }
    if (i + 1 >= argc) { usage(argv[0]); return 1; }
    const char *v = argv[++i];
    if (k == "--input") input = v;
    else if (k == "--type") type = v;
    else if (k == "--skip") skip = (unsigned)strtoul(v, nullptr, 10);
    else if (k == "--output") output = v;
    else if (k == "--device") device = atoi(v);
    else { usage(argv[0]); return 1; }
  }
  thv_format fmt;
  if (type == "csr") fmt = THV_FMT_CSR;
  else if (type == "csc") fmt = THV_FMT_CSC;
  else if (type == "wcsr") fmt = THV_FMT_WCSR;
  else {
    fprintf(stderr, "Error: --type must be csr, csc or wcsr (other converter outputs are not built)\n");
    return 1;
  }
  if (input.empty()) { usage(argv[0]); return 1; }
  if (output.empty()) {
    const size_t slash = input.find_last_of('/');
    const size_t dot = input.find_last_of('.');
    output = (dot != std::string::npos && (slash == std::string::npos || dot > slash)
                  ? input.substr(0, dot) : input) + "." + type;
  }
  printf("Converting to %s\n", type == "csr" ? "CSR" : type == "csc" ? "CSC" : "WCSR");
  uint64_t nv = 0, ne = 0;
  const thv_status s = thv_convert(input.c_str(), output.c_str(), fmt, skip, flags, device, &nv, &ne);
  if (s != THV_OK) {
    fprintf(stderr, "Error: %s\n", thv_last_error());
    return 1;
  }
  printf("Wrote %s: %llu vertices, %llu edges\n", output.c_str(), (unsigned long long)nv,
         (unsigned long long)ne);
  return 0;
}
