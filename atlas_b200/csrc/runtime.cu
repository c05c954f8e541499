// Runtime state of the library: device selection, one CUDA stream per host
// thread (replacing the reference's pthread pool, src/threads/), grow-only
// device/pinned buffer caches so a warm call performs no allocation, and
// error reporting.
#include <cstring>
#include <cstdarg>
#include <mutex>
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
  Buf dev[kNumSlots];
  Buf host[kNumSlots];
  ~ThreadState() {
    // buffers are left to process teardown (the CUDA context may already be
    // gone when thread-local destructors run at exit)
  }
};
thread_local ThreadState tl;
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

void *scratch(int slot, size_t bytes) {
  Buf &b = tl.dev[slot];
  if (bytes == 0) bytes = 16;
  if (b.n < bytes) {
    cudaStream_t st = stream();
    if (b.p) {
      ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
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
  Buf &b = tl.host[slot];
  if (bytes == 0) bytes = 16;
  if (b.n < bytes) {
    cudaStream_t st = stream();
    if (b.p) {
      ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
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
