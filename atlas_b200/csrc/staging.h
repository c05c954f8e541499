// Host/device staging helpers of the C ABI: drop-in entry points accept host
// or device pointers; host matrices are packed into cached device buffers.
#pragma once
#include <algorithm>
#include "common.cuh"

namespace atlb {

inline bool is_dev(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
struct DMat {
  T *d;
  long ld;
  bool in_place;
};

// Bring a rows x cols column-major host matrix (leading dimension ld) to the
// device; device pointers are used where they are.
template <typename T>
inline DMat<T> stage_in(int slot, const T *h, int rows, int cols, long ld, bool copy, cudaStream_t st) {
  if (is_dev(h)) return {(T *)h, ld, true};
  long dld = std::max(rows, 1);
  T *d = (T *)scratch(slot, sizeof(T) * (size_t)dld * std::max(cols, 1));
  if (copy && rows > 0 && cols > 0)
    ATLB_CUDA_CHECK(cudaMemcpy2DAsync(d, dld * sizeof(T), h, ld * sizeof(T), rows * sizeof(T),
                                      cols, cudaMemcpyHostToDevice, st));
  return {d, dld, false};
}

template <typename T>
inline void stage_out(T *h, long ld, const DMat<T> &m, int rows, int cols, cudaStream_t st) {
  if (m.in_place || rows <= 0 || cols <= 0) return;
  ATLB_CUDA_CHECK(cudaMemcpy2DAsync(h, ld * sizeof(T), m.d, m.ld * sizeof(T), rows * sizeof(T),
                                    cols, cudaMemcpyDeviceToHost, st));
}

template <typename T>
inline T *stage_vec_in(int slot, const T *h, int n, bool copy, cudaStream_t st) {
  if (is_dev(h)) return (T *)h;
  T *d = (T *)scratch(slot, sizeof(T) * std::max(n, 1));
  if (copy && n > 0)
    ATLB_CUDA_CHECK(cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
  return d;
}
template <typename T>
inline void stage_vec_out(T *h, const T *d, int n, cudaStream_t st) {
  if (h == d || n <= 0) return;
  ATLB_CUDA_CHECK(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, st));
}

}  // namespace atlb
