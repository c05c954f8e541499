// Runtime state of the library: device selection, one CUDA stream per host
// thread (replacing the reference's pthread pool, src/threads/), grow-only
// device/pinned buffer caches so a warm call performs no allocation, and
// error reporting.
#include <cstring>
#include <cstdarg>
#include <functional>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "../../include/atlas_b200.h"

namespace atlb {

namespace {
struct Buf {
  void *p = nullptr;
  size_t n = 0;
};
struct ThreadState {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t side = nullptr;
  cudaStream_t copy = nullptr;
  cudaEvent_t events[8] = {};
  std::vector<cudaEvent_t> chunk_events;
  Buf dev[2 * kNumSlots];   // second half: buffers of work on the side stream
  Buf host[2 * kNumSlots];
  ~ThreadState() {
    // buffers are left to process teardown (the CUDA context may already be
    // gone when thread-local destructors run at exit)
  }
};
thread_local ThreadState tl;
thread_local int tl_side = 0;                 // a SideScope is active on this thread
thread_local bool tl_capturing = false;       // a graph capture is recording on this thread
thread_local bool tl_capture_failed = false;  // ...and needed a workspace it could not grow
thread_local unsigned long long tl_scratch_gen = 0;  // bumps whenever a workspace moves
int g_device = -1;
int g_sms = 0;
std::mutex g_init_mu;
int g_err_mode = -1;  // 0: exit(-1) like cblas_xerbla, 1: return the error code
thread_local int tl_last_error = 0;
thread_local cudaError_t tl_cuda_error = cudaSuccess;

void ensure_device() {
  if (g_device >= 0) return;
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (g_device >= 0) return;
  int dev = 0;
  const char *e = getenv("ATLAS_B200_DEVICE");
  if (e) dev = atoi(e);
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    fprintf(stderr, "atlas_b200: no CUDA device available; this library has no CPU path\n");
    exit(-1);
  }
  ATLB_CUDA_CHECK(cudaSetDevice(dev));
  cudaDeviceProp prop;
  ATLB_CUDA_CHECK(cudaGetDeviceProperties(&prop, dev));
  g_sms = prop.multiProcessorCount;
  g_device = dev;
}
}  // namespace

void set_cuda_error(cudaError_t e) { tl_cuda_error = e; }

int num_sms() {
  ensure_device();
  return g_sms;
}

cudaStream_t stream() {
  ensure_device();
  if (!tl.stream) {
    ATLB_CUDA_CHECK(cudaSetDevice(g_device));
    ATLB_CUDA_CHECK(cudaStreamCreateWithFlags(&tl.stream, cudaStreamNonBlocking));
    tl.own_stream = true;
  }
  return tl.stream;
}

cudaStream_t side_stream() {
  ensure_device();
  if (!tl.side) {
    int least = 0, greatest = 0;
    ATLB_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    ATLB_CUDA_CHECK(cudaStreamCreateWithPriority(&tl.side, cudaStreamNonBlocking, greatest));
  }
  return tl.side;
}

cudaStream_t copy_stream() {
  ensure_device();
  if (!tl.copy) ATLB_CUDA_CHECK(cudaStreamCreateWithFlags(&tl.copy, cudaStreamNonBlocking));
  return tl.copy;
}

cudaEvent_t chunk_event(int i) {
  while ((int)tl.chunk_events.size() <= i) {
    cudaEvent_t e;
    ATLB_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    tl.chunk_events.push_back(e);
  }
  return tl.chunk_events[i];
}

cudaEvent_t side_event(int i) {
  if (!tl.events[i]) ATLB_CUDA_CHECK(cudaEventCreateWithFlags(&tl.events[i], cudaEventDisableTiming));
  return tl.events[i];
}

SideScope::SideScope() { tl_side = 1; }
SideScope::~SideScope() { tl_side = 0; }

namespace {
thread_local int tl_no_alloc = 0;
}
NoAllocScope::NoAllocScope() { tl_no_alloc++; }
NoAllocScope::~NoAllocScope() { tl_no_alloc--; }
bool no_alloc_active() { return tl_no_alloc > 0; }

namespace {
thread_local int tl_gemm_cap = 0;
}
GemmCtaCap::GemmCtaCap(int ctas) : prev(tl_gemm_cap) { tl_gemm_cap = ctas; }
GemmCtaCap::~GemmCtaCap() { tl_gemm_cap = prev; }
int gemm_cta_cap() { return tl_gemm_cap; }

void *scratch(int slot, size_t bytes) {
  Buf &b = tl.dev[slot + tl_side * kNumSlots];
  if (bytes == 0) bytes = 16;
  if (b.n < bytes && no_alloc_active()) return nullptr;
  if (b.n < bytes && tl_capturing) {
    // cannot allocate while recording a graph: the capture is abandoned and
    // the work re-run eagerly (the pointer returned here is never executed)
    tl_capture_failed = true;
    return b.p ? b.p : (void *)tl.dev;
  }
  if (b.n < bytes) {
    tl_scratch_gen++;
    cudaStream_t st = stream();
    if (b.p) {
      ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
      if (tl.side) ATLB_CUDA_CHECK(cudaStreamSynchronize(tl.side));
      ATLB_CUDA_CHECK(cudaFree(b.p));
    }
    size_t n = (bytes + (1 << 20) - 1) & ~((size_t)(1 << 20) - 1);
    if (cudaMalloc(&b.p, n) != cudaSuccess) {
      cudaGetLastError();
      fprintf(stderr, "atlas_b200: device allocation of %zu bytes failed\n", n);
      b.p = nullptr;
      b.n = 0;
      return nullptr;
    }
    b.n = n;
  }
  return b.p;
}

void *pinned(int slot, size_t bytes) {
  Buf &b = tl.host[slot + tl_side * kNumSlots];
  if (bytes == 0) bytes = 16;
  if (b.n < bytes && no_alloc_active()) return nullptr;
  if (b.n < bytes && tl_capturing) {
    tl_capture_failed = true;
    return b.p ? b.p : (void *)tl.host;
  }
  if (b.n < bytes) {
    cudaStream_t st = stream();
    if (b.p) {
      ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
      if (tl.side) ATLB_CUDA_CHECK(cudaStreamSynchronize(tl.side));
      ATLB_CUDA_CHECK(cudaFreeHost(b.p));
    }
    size_t n = (bytes + (1 << 20) - 1) & ~((size_t)(1 << 20) - 1);
    if (cudaMallocHost(&b.p, n) != cudaSuccess) {
      cudaGetLastError();
      b.p = nullptr;
      b.n = 0;
      return nullptr;
    }
    b.n = n;
  }
  return b.p;
}

// ---------------------------------------------------------------- graphs
namespace {
struct GraphEntry {
  std::vector<unsigned long long> key;
  cudaGraphExec_t exec;
  unsigned long long gen;
  unsigned long long last_use;
};
thread_local std::vector<GraphEntry> tl_graphs;
thread_local std::vector<std::vector<unsigned long long>> tl_seen;
thread_local unsigned long long tl_clock = 0;
constexpr size_t kMaxGraphs = 24;

bool graphs_enabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("ATLAS_B200_GRAPHS");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}
}  // namespace

void run_graph(const std::vector<unsigned long long> &key, cudaStream_t st,
               const std::function<void()> &enqueue) {
  if (!graphs_enabled()) { enqueue(); return; }
  tl_clock++;
  for (auto &g : tl_graphs) {
    if (g.key == key) {
      if (g.gen == tl_scratch_gen) {
        g.last_use = tl_clock;
        ATLB_CUDA_CHECK(cudaGraphLaunch(g.exec, st));
        return;
      }
      cudaGraphExecDestroy(g.exec);  // a workspace moved since the capture
      g = tl_graphs.back();
      tl_graphs.pop_back();
      break;
    }
  }
  bool seen = false;
  for (auto &k : tl_seen) if (k == key) { seen = true; break; }
  if (!seen) {  // first call: eager (sizes every workspace, sets kernel attributes)
    if (tl_seen.size() > 64) tl_seen.erase(tl_seen.begin());
    tl_seen.push_back(key);
    enqueue();
    return;
  }
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    enqueue();  // the caller is capturing already: just record into its graph
    return;
  }
  cudaGraph_t graph = nullptr;
  tl_capturing = true;
  tl_capture_failed = false;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue();
    e = cudaStreamEndCapture(st, &graph);
  }
  tl_capturing = false;
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess && !tl_capture_failed && graph)
    // keep the side stream's priority inside the graph (look-ahead panels)
    e = cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess || tl_capture_failed || !exec) {
    cudaGetLastError();
    if (exec) cudaGraphExecDestroy(exec);
    enqueue();
    return;
  }
  if (tl_graphs.size() >= kMaxGraphs) {  // evict the least recently used
    size_t lru = 0;
    for (size_t i = 1; i < tl_graphs.size(); i++)
      if (tl_graphs[i].last_use < tl_graphs[lru].last_use) lru = i;
    cudaGraphExecDestroy(tl_graphs[lru].exec);
    tl_graphs[lru] = tl_graphs.back();
    tl_graphs.pop_back();
  }
  tl_graphs.push_back({key, exec, tl_scratch_gen, tl_clock});
  ATLB_CUDA_CHECK(cudaGraphLaunch(exec, st));
}

int err_mode() {
  if (g_err_mode < 0) {
    const char *e = getenv("ATLAS_B200_XERBLA");
    g_err_mode = (e && strcmp(e, "return") == 0) ? 1 : 0;
  }
  return g_err_mode;
}

// Report bad argument `pos` of `rout` the way cblas_xerbla does
// (interfaces/blas/C/src/cblas_xerbla.c:13-28): message on stderr, then
// exit(-1) -- unless the caller switched to return mode.
void xerbla(int pos, const char *rout) {
  if (pos) fprintf(stderr, "Parameter %d to routine %s was incorrect\n", pos, rout);
  tl_last_error = -pos;
  if (err_mode() == 0) exit(-1);
}

}  // namespace atlb

using namespace atlb;

extern "C" {

int atlb_init(int device) {
  if (device >= 0) {
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_device < 0) {
      int n = 0;
      if (cudaGetDeviceCount(&n) != cudaSuccess || device >= n) return -1;
      if (cudaSetDevice(device) != cudaSuccess) return -1;
      cudaDeviceProp prop;
      cudaGetDeviceProperties(&prop, device);
      g_sms = prop.multiProcessorCount;
      g_device = device;
    }
  }
  stream();
  return g_device;
}

void atlb_set_error_mode(int mode) { g_err_mode = mode ? 1 : 0; }
int atlb_get_error_mode(void) { return err_mode(); }
int atlb_last_error(void) { return tl_last_error; }
int atlb_last_cuda_error(void) { return (int)tl_cuda_error; }

void *atlb_get_stream(void) { return (void *)stream(); }
void atlb_set_stream(void *s) {
  ensure_device();
  if (tl.stream && tl.own_stream) {
    cudaStreamSynchronize(tl.stream);
    cudaStreamDestroy(tl.stream);
  }
  tl.stream = (cudaStream_t)s;
  tl.own_stream = false;
  if (!s) stream();
}
int atlb_sync(void) {
  cudaError_t e = cudaStreamSynchronize(stream());
  if (e != cudaSuccess) tl_cuda_error = e;
  return (int)e;
}

void cblas_xerbla(int p, const char *rout, const char *form, ...) {
  va_list ap;
  va_start(ap, form);
  if (p) fprintf(stderr, "Parameter %d to routine %s was incorrect\n", p, rout);
  vfprintf(stderr, form, ap);
  va_end(ap);
  tl_last_error = -p;
  if (err_mode() == 0) exit(-1);
}

int cblas_errprn(int ierr, int info, char *form, ...) {
  va_list ap;
  va_start(ap, form);
  vfprintf(stderr, form, ap);
  va_end(ap);
  return ierr < info ? ierr : info;
}

}  // extern "C"
