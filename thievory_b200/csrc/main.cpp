// ./main -- drop-in for the reference CLI (src/main.cu:44-225).
//
// Same flags and defaults: --input, --algo bfs|cc|sssp|pr (bfs),
// --edgeSize 4|8 (4), --type push|pull (push), --source (1), --runs (1),
// --gpus (0), --device (0).  Same output: "Execution time: X ms" per run,
// "Average execution time: X ms", and results/values.bin (u32 per vertex, or
// double for PageRank; written only when results/ exists, as the reference
// does).  Differences, by design:
//   --gpus must be 0 (one GPU, no neighbour-GPU stealing);
//   --edgeSize 8 reads WCSR ({u32 dst, u32 w} edges) instead of being a stub;
//   SSSP with --edgeSize 4 uses the weight section of the .csr file;
//   PageRank is the fixed-iteration FP32 method (damping 0.85, 20 iterations,
//   dangling mass redistributed);
//   no nvidia-smi / NUMA probing; errors are reported, with exit code 1.
// Extra flags: --hbm-budget <bytes|N%|NK|NM|NG>, --block-bytes <bytes|NM>,
//   --placement densest|prefix, --pr-iters N, --values <path>,
//   --pr-semantics fixed|reference (fixed: FP32, --pr-iters iterations;
//   reference: the reference engine's FP64 rounds to a 1e-3 tolerance).
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "thv.h"

static void usage(const char *prog) {
  printf("Usage: %s\n", prog);
  printf("Options:\n");
  printf("  --input : path to the graph (.csr, .csc for pull PageRank, .wcsr for --edgeSize 8)\n");
  printf("  --algo : {'bfs', 'cc', 'pr', 'sssp'} (default = 'bfs')\n");
  printf("  --edgeSize : {4, 8} (default = 4)\n");
  printf("  --type : PageRank type {'push', 'pull'} (default = 'push')\n");
  printf("  --source : source vertex (default = 1)\n");
  printf("  --runs : number of runs (default = 1)\n");
  printf("  --gpus : neighbour GPUs, must be 0 (default = 0)\n");
  printf("  --device : CUDA device (default = 0)\n");
  printf("  --hbm-budget : resident edge bytes (e.g. 2G, 40%%; default: all that fit)\n");
  printf("  --block-bytes : edge block size (default 64M)\n");
  printf("  --placement : densest|prefix (default densest)\n");
  printf("  --symmetric : 1 = the graph has every reverse edge (CC by union-find)\n");
  printf("  --pr-iters : PageRank iterations (default 20)\n");
  printf("  --pr-semantics : fixed|reference (default fixed; reference = FP64 to 1e-3)\n");
  printf("  --values : output path (default results/values.bin)\n");
}

static bool parse_size(const char *s, uint64_t total, uint64_t *out) {
  char *end = nullptr;
  const double x = strtod(s, &end);
  if (end == s || x < 0) return false;
  double mul = 1;
  if (*end == '%') { *out = (uint64_t)(x / 100.0 * (double)total); return true; }
  if (*end == 'K' || *end == 'k') mul = 1024.0;
  else if (*end == 'M' || *end == 'm') mul = 1024.0 * 1024;
  else if (*end == 'G' || *end == 'g') mul = 1024.0 * 1024 * 1024;
  else if (*end != 0) return false;
  *out = (uint64_t)(x * mul);
  return true;
}

static int die(const char *what, thv_status s) {
  fprintf(stderr, "Error: %s: %s (%s)\n", what, thv_status_str(s), thv_last_error());
  return 1;
}

int main(int argc, char **argv) {
  std::string input, algo = "bfs", type = "push", budget, block, placement = "densest";
  std::string pr_semantics = "fixed";
  std::string values_path = "results/values.bin";
  unsigned edge_size = 4, source = 1, runs = 1, gpus = 0, pr_iters = 20;
  int device = 0;
  bool has_input = false, symmetric = false;
  for (int i = 1; i + 1 < argc; i += 2) {
    const char *k = argv[i], *v = argv[i + 1];
    if (!strcmp(k, "--input")) { input = v; has_input = true; }
    else if (!strcmp(k, "--algo")) algo = v;
    else if (!strcmp(k, "--edgeSize")) edge_size = (unsigned)atoi(v);
    else if (!strcmp(k, "--type")) type = v;
    else if (!strcmp(k, "--source")) source = (unsigned)strtoul(v, nullptr, 10);
    else if (!strcmp(k, "--runs")) runs = (unsigned)atoi(v);
    else if (!strcmp(k, "--gpus")) gpus = (unsigned)atoi(v);
    else if (!strcmp(k, "--device")) device = atoi(v);
    else if (!strcmp(k, "--hbm-budget")) budget = v;
    else if (!strcmp(k, "--block-bytes")) block = v;
    else if (!strcmp(k, "--placement")) placement = v;
    else if (!strcmp(k, "--pr-iters")) pr_iters = (unsigned)atoi(v);
    else if (!strcmp(k, "--pr-semantics")) pr_semantics = v;
    else if (!strcmp(k, "--values")) values_path = v;
    else if (!strcmp(k, "--symmetric")) symmetric = atoi(v) != 0;
    else { fprintf(stderr, "Error: unknown flag %s\n", k); usage(argv[0]); return 1; }
  }
  if (!has_input) { usage(argv[0]); return 0; }
  if (gpus != 0) {
    fprintf(stderr, "Error: --gpus %u: this engine runs on one GPU (--gpus 0)\n", gpus);
    return 1;
  }
  if (edge_size != 4 && edge_size != 8) {
    fprintf(stderr, "Error: wrong --edgeSize\n");
    usage(argv[0]);
    return 1;
  }
  thv_algo a;
  thv_format fmt;
  uint32_t flags = 0;
  if (algo == "bfs" || algo == "cc") {
    a = algo == "bfs" ? THV_ALGO_BFS : THV_ALGO_CC;
    fmt = edge_size == 8 ? THV_FMT_WCSR : THV_FMT_CSR;
  } else if (algo == "sssp") {
    a = THV_ALGO_SSSP;
    fmt = edge_size == 8 ? THV_FMT_WCSR : THV_FMT_CSR;
    flags = THV_OPEN_WEIGHTS;
  } else if (algo == "pr") {
    if (edge_size == 8 || type == "pull") { a = THV_ALGO_PR_PULL; fmt = THV_FMT_CSC; }
    else if (type == "push") { a = THV_ALGO_PR_PUSH; fmt = THV_FMT_CSR; }
    else { fprintf(stderr, "Error: wrong --type\n"); usage(argv[0]); return 1; }
  } else {
    usage(argv[0]);
    return 1;
  }
  printf("Running %s with edge size of %uB on device %d\n", algo.c_str(), edge_size, device);
  if (a == THV_ALGO_BFS || a == THV_ALGO_SSSP) printf("Source vertex is: %u\n", source);

  thv_graph *g = nullptr;
  thv_status s = thv_open(input.c_str(), fmt, flags, device, &g);
  if (s != THV_OK) return die("open", s);
  if (symmetric) thv_set_symmetric(g, 1);  // CC: sampling union-find
  thv_graph_info info{};
  thv_info(g, &info);
  printf("Num Vertices: %llu\n", (unsigned long long)info.nv);
  printf("Num Edges: %llu\n", (unsigned long long)info.ne);

  thv_plan_opts po{};
  po.hbm_budget_bytes = UINT64_MAX;
  po.block_bytes = 0;
  po.policy = placement == "prefix" ? THV_PLACE_PREFIX : THV_PLACE_DENSEST;
  // PageRank reads whole blocks: give the whole budget to blocks
  if (a == THV_ALGO_PR_PULL || a == THV_ALGO_PR_PUSH) po.small_list_degree = 1;
  const uint64_t edge_bytes = info.ne * info.esz;
  if (!budget.empty() && !parse_size(budget.c_str(), edge_bytes, &po.hbm_budget_bytes)) {
    fprintf(stderr, "Error: bad --hbm-budget %s\n", budget.c_str());
    thv_close(g);
    return 1;
  }
  if (!block.empty() && !parse_size(block.c_str(), edge_bytes, &po.block_bytes)) {
    fprintf(stderr, "Error: bad --block-bytes %s\n", block.c_str());
    thv_close(g);
    return 1;
  }
  s = thv_plan(g, &po);
  if (s != THV_OK) { thv_close(g); return die("plan", s); }
  thv_plan_info pi{};
  thv_get_plan(g, &pi);
  printf("Number of partitions: %llu (resident %llu)\n",
         (unsigned long long)pi.num_blocks, (unsigned long long)pi.resident_blocks);
  printf("Resident edge bytes: %llu, host (zero-copy) edge bytes: %llu\n",
         (unsigned long long)pi.resident_edge_bytes, (unsigned long long)pi.host_edge_bytes);
  if (pi.small_list_degree)
    printf("Small lists (degree < %llu) cached in HBM: %llu vertices, %llu bytes\n",
           (unsigned long long)pi.small_list_degree, (unsigned long long)pi.small_list_vertices,
           (unsigned long long)pi.small_list_bytes);

  thv_run_opts ro{};
  ro.source = source;
  ro.pr_iters = pr_iters;
  if (pr_semantics == "reference") {
    ro.flags |= THV_RUN_PR_REFERENCE;
    ro.pr_iters = 0;
  } else if (pr_semantics != "fixed") {
    fprintf(stderr, "Error: wrong --pr-semantics\n");
    thv_close(g);
    return 1;
  }
  double total_ms = 0;
  thv_stats st{};
  for (unsigned r = 0; r < runs; r++) {
    s = thv_run(g, a, &ro, nullptr, &st);
    if (s != THV_OK) { thv_close(g); return die("run", s); }
    printf("Execution time: : %g ms\n", st.wall_ms);
    total_ms += st.wall_ms;
  }
  if (runs) {
    printf("Average execution time: %g ms\n", total_ms / runs);
    printf("Edges scanned: %llu, link bytes: %llu, HBM edge bytes: %llu, iterations: %llu\n",
           (unsigned long long)st.edges_expanded, (unsigned long long)st.link_edge_bytes,
           (unsigned long long)st.hbm_edge_bytes, (unsigned long long)st.iterations);
    const bool pr = a == THV_ALGO_PR_PUSH || a == THV_ALGO_PR_PULL;
    const size_t esz = pr ? 8 : 4;
    std::vector<char> vals(info.nv * esz + 8);
    s = thv_values(g, vals.data());
    if (s != THV_OK) { thv_close(g); return die("values", s); }
    // the reference skips the dump silently when results/ is missing
    FILE *f = fopen(values_path.c_str(), "wb");
    if (f) {
      fclose(f);
      s = thv_write_values(values_path.c_str(), vals.data(), info.nv, (uint32_t)esz);
      if (s != THV_OK) { thv_close(g); return die("write values", s); }
    }
  }
  thv_close(g);
  return 0;
}
