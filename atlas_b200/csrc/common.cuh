// Shared helpers for the sm_100a kernels and their host drivers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <vector>

#define ATLB_CUDA_CHECK(expr)                                                  \
  do {                                                                         \
    cudaError_t e__ = (expr);                                                  \
    if (e__ != cudaSuccess) {                                                  \
      fprintf(stderr, "atlas_b200: CUDA error %s at %s:%d: %s\n",             \
              cudaGetErrorName(e__), __FILE__, __LINE__,                       \
              cudaGetErrorString(e__));                                        \
      atlb::set_cuda_error(e__);                                               \
    }                                                                          \
  } while (0)

namespace atlb {

// Enum values of the CBLAS interface (include/cblas.h:5-10 of the reference).
enum { kRowMajor = 101, kColMajor = 102 };
enum { kNoTrans = 111, kTrans = 112, kConjTrans = 113 };
enum { kUpper = 121, kLower = 122 };
enum { kNonUnit = 131, kUnit = 132 };
enum { kLeft = 141, kRight = 142 };

void set_cuda_error(cudaError_t e);
cudaStream_t stream();           // the library's stream for the calling thread
int num_sms();

// Device memory cache: grow-only buffers keyed by slot, reused across calls
// so the hot path performs no cudaMalloc once warm.
void *scratch(int slot, size_t bytes);
void *pinned(int slot, size_t bytes);
// A second, high-priority stream per host thread for work that runs beside
// the main stream (look-ahead panels).  While a SideScope is alive on a
// thread, scratch() and pinned() hand out a second set of buffers, so work
// enqueued on the two streams never shares a workspace.
cudaStream_t side_stream();
cudaEvent_t side_event(int i);  // eight reusable events per thread (i < 8)
// A third stream per host thread for host-to-device copies that overlap the
// factorization (streamed inputs), and a growable set of events for them.
cudaStream_t copy_stream();
cudaEvent_t chunk_event(int i);
struct SideScope {
  SideScope();
  ~SideScope();
};
// While a NoAllocScope is alive on a thread, scratch() and pinned() never
// allocate (they return nullptr instead of growing a buffer) and the GEMM
// driver does not take its split-K path, which needs a workspace.
struct NoAllocScope {
  NoAllocScope();
  ~NoAllocScope();
};
bool no_alloc_active();
// While a GemmCtaCap is alive on a thread, large DGEMMs run on at most that
// many CTAs (0: no cap).
struct GemmCtaCap {
  explicit GemmCtaCap(int ctas);
  ~GemmCtaCap();
  int prev;
};
int gemm_cta_cap();
enum ScratchSlot {
  kSlotA = 0, kSlotB, kSlotC, kSlotIpiv, kSlotTau, kSlotWork, kSlotWork2,
  kSlotInfo, kSlotMixedA, kSlotMixedR, kSlotMixedX, kSlotMixedD,
  kSlotOzA, kSlotOzB, kSlotOzScale, kSlotBatch0, kSlotBatch1, kSlotBatch2,
  kSlotBatch3, kSlotAdj0, kSlotAdj1, kSlotAdj2, kSlotTc0, kSlotTc1, kSlotTrsmW, kSlotTrsvCtl, kSlotLaswp,
  kSlotMixedWL, kSlotMixedWU, kSlotMixedPerm, kSlotGemmSplit, kSlotPermPlan,
  kSlotQrApply, kSlotExt0, kSlotExt1, kSlotExt2, kSlotExt3, kSlotAdjProbs, kSlotKrylov, kSlotKrylovH,
  kSlotStreamPerm, kSlotStreamTmp, kNumSlots
};

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// Tunable driver parameters (tuning.cu; chosen by atlas_b200/tune.py).
enum TuneParam {
  kTuneGetrfNB = 0, kTunePotrfNB, kTuneGemmGroup, kTuneSplitK, kTuneLookahead, kTuneTcMinWorkLog2,
  kTuneLookaheadReserve, kTuneSgetrfNB, kTuneQrNB, kTuneBatchPosvSmall, kTuneBatchPosvPW,
  kTuneMixedKrylov, kNumTune
};
int tune(int p);
int tune_generation();  // bumps whenever a parameter changes (part of graph keys)

// Replay cache for launch sequences that depend only on their arguments
// (sizes, pointers, stream): the first call with a key runs `enqueue`
// eagerly (sizing every workspace), the second captures it into a CUDA graph,
// later calls launch the graph.  A workspace that moves invalidates the
// cached graphs; ATLAS_B200_GRAPHS=0 turns the cache off.
void run_graph(const std::vector<unsigned long long> &key, cudaStream_t st,
               const std::function<void()> &enqueue);

}  // namespace atlb

// ---------------------------------------------------------------------------
// Device helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
  uint32_t s = smem_u32(smem);
  int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
  uint32_t s = smem_u32(smem);
  int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool pred) {
  uint32_t s = smem_u32(smem);
  int n = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }
