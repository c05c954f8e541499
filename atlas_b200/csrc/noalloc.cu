// Triangular solve that allocates no device memory.
//
// atlb_dtrsm_dev takes its workspace (the inverted 64x64 diagonal blocks of
// the triangle) from the library's buffer cache, which calls cudaMalloc the
// first time a size is seen.  Some callers cannot allow that: applications
// whose device memory is owned by their own pool or framework allocator and
// must not change behind its back, and programs with a fixed memory budget
// that is checked up front.  This entry point serves them: its workspace is
// one array compiled into the library, sized for triangles of order up to
// kNoAllocMaxN, which every GPU that loads the library holds until the
// process exits (2 MiB).
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side placeholder), so the device address is looked up with
// cudaGetSymbolAddress once per device, with the library's device (the one
// its stream belongs to) made current for the lookup, on the first call that
// runs on that device.  Make that first call before any stream capture
// begins.  All calls share the one array: calls that overlap on the GPU (two
// streams, two host threads) race on it, so serialize them.  Every call
// rewrites all of the array it reads, so nothing left by an earlier call is
// used.
#include <algorithm>
#include <mutex>
#include "common.cuh"
#include "kernels.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

constexpr int kLeafN = 64;            // order of the inverted diagonal blocks
constexpr int kNoAllocMaxN = 4096;    // largest triangle this entry point solves with
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_trsm_w[(kNoAllocMaxN / kLeafN) * kLeafN * kLeafN];

std::mutex g_addr_mu;
double *g_addr[kMaxDevices] = {};

// Device address of the array on device `dev` (nullptr on failure).  The
// lookup runs with `dev` current and puts the caller's current device back.
double *workspace_address(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_trsm_w);
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      fprintf(stderr, "atlas_b200: atlb_dtrsm_dev_noalloc: cudaGetSymbolAddress failed: %s\n",
              cudaGetErrorString(e));
      return nullptr;
    }
    g_addr[dev] = static_cast<double *>(p);
  }
  return g_addr[dev];
}

}  // namespace
}  // namespace atlb

using namespace atlb;

extern "C" int atlb_dtrsm_dev_noalloc(int Side, int Uplo, int TA, int Diag, int M, int N, double alpha,
                                      const double *A, int lda, double *B, int ldb) {
  if (Side != kLeft && Side != kRight) return -1;
  if (Uplo != kUpper && Uplo != kLower) return -2;
  if (TA != kNoTrans && TA != kTrans && TA != kConjTrans) return -3;
  if (Diag != kUnit && Diag != kNonUnit) return -4;
  if (M < 0) return -5;
  if (N < 0) return -6;
  const int order = Side == kLeft ? M : N;
  if (order > kNoAllocMaxN) {
    fprintf(stderr,
            "atlas_b200: atlb_dtrsm_dev_noalloc: triangle of order %d exceeds the fixed workspace "
            "(order <= %d); use atlb_dtrsm_dev\n",
            order, kNoAllocMaxN);
    return Side == kLeft ? -5 : -6;
  }
  if (lda < std::max(1, order)) return -9;
  if (ldb < std::max(1, M)) return -11;
  if (M == 0 || N == 0) return 0;
  // The solve runs on the library's stream, which belongs to the library's
  // device (atlb_init / ATLAS_B200_DEVICE), not necessarily to this host
  // thread's current device: the array's address is taken on that device.
  cudaStream_t st = stream();
  double *W = workspace_address(atlb_init(-1));
  if (!W) return -100;
  NoAllocScope guard;  // the GEMMs inside the solve must not take a workspace either
  trsm_impl<double>(Side, Uplo, TA == kNoTrans ? kNoTrans : kTrans, Diag, M, N, alpha, A, lda, B, ldb,
                    st, nullptr, W);
  return 0;
}
