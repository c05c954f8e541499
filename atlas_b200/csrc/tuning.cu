// Tunable parameters of the drivers, in the spirit of ATLAS's install-time
// search (tune/blas/gemm/gmmsearch.c): atlas_b200/tune.py times the
// candidates of each parameter on the GPU and writes the winners to
// tuning.conf beside the library; the library reads that file the first time
// a parameter is used.  ATLAS_B200_TUNE_FILE names another file; "none"
// skips the file (defaults only).  atlb_tune_set changes a value at run time
// (the tuner's search uses it).
//
// File format: one "name value" pair per line, '#' starts a comment.
#include <atomic>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <string>
#include "common.cuh"
#include "kernels.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

struct TuneDef {
  const char *name;
  int def, lo, hi, step;  // value is clamped to [lo, hi] and rounded down to a multiple of step
};
const TuneDef kDefs[kNumTune] = {
    {"getrf_nb", 256, 64, 256, 32},           // outer LU block (leaf panels are 32 wide)
    {"potrf_nb", 256, 64, 16384, 64},         // outer Cholesky block (leaves are 128 wide; >= N: pure recursion)
    {"dgemm_group", 8, 1, 64, 1},             // DGEMM rasterisation: tile rows sharing B panels
    {"dgemm_splitk", 1, 0, 1, 1},             // split K when the output has too few tiles
    {"lookahead", 1, 0, 1, 1},                // depth-one look-ahead in getrf / potrf
    {"mixed_tc_min_work_log2", 31, 16, 40, 1},  // mixed solvers: M*N*K below 2^x runs on FP32 FMA
    {"lookahead_reserve_sms", 0, 0, 96, 1},   // SMs the trailing-update DGEMM leaves to the look-ahead panel
    {"sgetrf_nb", 256, 64, 256, 32},          // outer LU block of the FP32 factorization (mixed solvers)
    {"qr_nb", 128, 32, 256, 32},              // QR panel width (ilaenv's NB for geqrf; > 128: two halves)
    {"batch_posv_small", 64, 32, 128, 16},    // batched Cholesky: orders <= this factor whole in shared memory
    {"batch_posv_pw", 16, 16, 64, 16},        // batched Cholesky: panel width above that order
    {"mixed_krylov", 1, 0, 2, 1},             // mixed solvers: 0 plain refinement, 1 GMRES-IR once plain stalls
                                              // (from the start for BF16), 2 GMRES-IR from the start
};

std::atomic<int> g_val[kNumTune];
std::atomic<int> g_gen{0};
std::once_flag g_once;

int clampv(int p, int v) {
  const TuneDef &d = kDefs[p];
  v = std::max(d.lo, std::min(d.hi, v));
  return v / d.step * d.step;
}

int find(const char *name) {
  for (int p = 0; p < kNumTune; p++)
    if (strcmp(kDefs[p].name, name) == 0) return p;
  return -1;
}

int load_file(const char *path) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char line[256];
  int n = 0;
  while (fgets(line, sizeof line, f)) {
    char *hash = strchr(line, '#');
    if (hash) *hash = 0;
    char name[128];
    int v;
    if (sscanf(line, "%127s %d", name, &v) == 2) {
      const int p = find(name);
      if (p >= 0) { g_val[p] = clampv(p, v); n++; }
    }
  }
  fclose(f);
  g_gen++;
  return n;
}

std::string default_path() {
  const char *e = getenv("ATLAS_B200_TUNE_FILE");
  if (e) return e;
  Dl_info info;
  if (dladdr((void *)&load_file, &info) && info.dli_fname) {
    std::string so = info.dli_fname;
    const size_t slash = so.rfind('/');
    return (slash == std::string::npos ? std::string(".") : so.substr(0, slash)) + "/tuning.conf";
  }
  return "tuning.conf";
}

void init() {
  std::call_once(g_once, [] {
    for (int p = 0; p < kNumTune; p++) g_val[p] = kDefs[p].def;
    const char *la = getenv("ATLAS_B200_LOOKAHEAD");
    const std::string path = default_path();
    if (path != "none") load_file(path.c_str());
    if (la) g_val[kTuneLookahead] = la[0] == '0' ? 0 : 1;
  });
}

}  // namespace

int tune(int p) {
  init();
  return g_val[p].load(std::memory_order_relaxed);
}

int tune_generation() {
  init();
  return g_gen.load(std::memory_order_relaxed);
}

}  // namespace atlb

using namespace atlb;

extern "C" {

int atlb_tune_get(const char *name) {
  init();
  const int p = name ? find(name) : -1;
  return p < 0 ? INT_MIN : g_val[p].load();
}

int atlb_tune_set(const char *name, int value) {
  init();
  const int p = name ? find(name) : -1;
  if (p < 0) return -1;
  g_val[p] = clampv(p, value);
  g_gen++;
  return g_val[p].load();
}

int atlb_tune_load(const char *path) {
  init();
  const std::string pth = path ? std::string(path) : default_path();
  return load_file(pth.c_str());
}

int atlb_tune_count(void) { return kNumTune; }

const char *atlb_tune_name(int i) { return (i >= 0 && i < kNumTune) ? kDefs[i].name : nullptr; }

}  // extern "C"
