// Wrapper entry point for building the reference engine (test infrastructure,
// output in oracle/_ref/thv_ref).  It replaces the reference's src/main.cu
// only to (1) skip the nvidia-smi NUMA probe (src/main.cu:118-147), (2) fix
// --gpus 0, and (3) optionally hold an HBM ballast so the reference's own
// static-edge budget -- 90% (45% for SSSP) of the free memory it sees in
// SetNumStaticEdges, src/graph.cuh:306-341 -- comes out near a requested
// byte count.  The engine code itself is the unmodified reference, compiled
// from its own sources; it dispatches exactly as src/main.cu:152-220.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>

#include "bfs/bfs.cuh"
#include "cc/cc.cuh"
#include "pr/pr.cuh"
#include "sssp/sssp.cuh"

// Device bytes the reference allocates before SetNumStaticEdges
// (src/graph.cuh:344-611, nNGPUs = 0).
static size_t ref_preallocs(const std::string &algo, const std::string &type,
                            uint64_t nv) {
  const size_t mb2 = 2u << 20;
  size_t b = 8 * (nv + 1) + 3 * 4 * nv + 4 * nv + nv;  // offsets, lists, flags, inStatic
  if (algo == "pr") {
    b += 8 * nv;
    if (type == "push") b += 2 * 8 * (nv + 1);
    else b += 4 * nv + 8 * nv;
  } else {
    b += 4 * nv;
  }
  const size_t filter = (size_t)N_TARGET_FILTER_STREAMS * (size_t)(PARTITION_SIZE_MB / 4) * 8;
  b += filter;
  if (algo == "sssp") b += filter;
  return b + 24 * mb2;
}

int main(int argc, char **argv) {
  cudaFree(0);
  cudaSetDevice(0);
  std::string path, algo = "bfs", type = "push";
  uint32 edge = 4, src = 1, runs = 1;
  long long budget = -1;
  for (int i = 1; i + 1 < argc; i += 2) {
    if (!strcmp(argv[i], "--input")) path = argv[i + 1];
    else if (!strcmp(argv[i], "--algo")) algo = argv[i + 1];
    else if (!strcmp(argv[i], "--edgeSize")) edge = atoi(argv[i + 1]);
    else if (!strcmp(argv[i], "--type")) type = argv[i + 1];
    else if (!strcmp(argv[i], "--source")) src = atoi(argv[i + 1]);
    else if (!strcmp(argv[i], "--runs")) runs = atoi(argv[i + 1]);
    else if (!strcmp(argv[i], "--static-budget")) budget = atoll(argv[i + 1]);
  }
  if (path.empty()) return 0;
  void *ballast = nullptr;
  if (budget >= 0) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); return 1; }
    uint64_t hdr[2] = {0, 0};
    if (fread(hdr, 8, 2, f) != 2) { fclose(f); return 1; }
    fclose(f);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const double frac = algo == "sssp" ? 0.45 : 0.9;
    const size_t want_free = ref_preallocs(algo, type, hdr[0]) + (size_t)(budget / frac);
    if (fr > want_free + (64u << 20)) {
      const size_t bal = fr - want_free;
      if (cudaMalloc(&ballast, bal) != cudaSuccess) { fprintf(stderr, "ballast failed\n"); return 1; }
      printf("Ballast bytes: %zu\n", bal);
    }
  }
  std::unordered_map<int, int> numa = {{0, 0}};
  if (algo == "bfs") {
    if (edge == 4) BFS32(path, src, runs, 0, numa);
    else BFS64(path, src, runs);
  } else if (algo == "cc") {
    if (edge == 4) CC32(path, runs, 0, numa);
    else CC64(path, runs);
  } else if (algo == "sssp") {
    if (edge == 4) SSSP32(path, src, runs, 0, numa);
    else SSSP64(path, src, runs);
  } else if (algo == "pr") {
    if (edge == 4 && type == "push") PR32_PUSH(path, runs, 0, numa);
    else PR32(path, runs, 0, numa);
  }
  // the reference checks no launch; report the context's state after the run
  const cudaError_t sync = cudaDeviceSynchronize();
  const cudaError_t last = cudaGetLastError();
  printf("Post-run CUDA status: sync=%s last=%s\n", cudaGetErrorString(sync),
         cudaGetErrorString(last));
  if (ballast) cudaFree(ballast);
  return sync == cudaSuccess && last == cudaSuccess ? 0 : 2;
}
