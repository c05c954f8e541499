// Triangular solve for a few right-hand sides (NRHS <= 8) in ONE launch.
//
// The recursive TRSM (trsm.cu) issues ~2n/64 launches, which for one
// right-hand side is all latency.  Here one CTA owns one 64-row block of the
// solution: it takes a ticket from an atomic counter (tickets are handed out
// in launch order, so every block it depends on is owned by a CTA that is
// already running and never waits on it), accumulates the products with the
// solved blocks as their "done" flags appear, multiplies by the inverted
// diagonal block (trinv_kernel's W) and publishes its block.  Every wait on a
// flag is bounded: after ~1 s the kernel records an error in *err and stops
// waiting (the result is then wrong but the GPU is released).  The launcher
// clears the ticket counter and the flags before each launch.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int BS = 64;

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T, int NR>
__global__ void __launch_bounds__(256)
trsv_kernel(int n, int nrhs, const T *__restrict__ Tp, long tr, long tc, int lower,
            const T *__restrict__ W, T *X, long ldx, int *counter, int *flags, int epoch, int *err) {
  extern __shared__ __align__(16) unsigned char trsv_smem[];
  T(*sW)[BS + 1] = reinterpret_cast<T(*)[BS + 1]>(trsv_smem);  // inverse of the diagonal block
  __shared__ T sacc[4][BS][NR];
  __shared__ T sx[BS][NR];
  __shared__ T sb[BS][NR];      // this block's right-hand side
  __shared__ int s_bi;
  const int tid = threadIdx.x, lane = tid & 31, nb = (n + BS - 1) / BS;
  if (tid == 0) {
    const int t = atomicAdd(counter, 1);
    s_bi = lower ? t : nb - 1 - t;
  }
  __syncthreads();
  const int bi = s_bi, r0 = bi * BS, rows = min(BS, n - r0);
  // everything that does not depend on other blocks is fetched first
  const T *Wb = W + (long)bi * BS * BS;
  for (int idx = tid; idx < BS * BS; idx += 256) sW[idx % BS][idx / BS] = Wb[idx];
  for (int idx = tid; idx < BS * NR; idx += 256) {
    const int rr = idx % BS, q = idx / BS;
    sb[rr][q] = (rr < rows && q < nrhs) ? X[r0 + rr + (long)q * ldx] : T(0);
  }
  // thread (r, part): row r of the block, columns part, part+4, ... of each
  // solved block; the next block's 16 matrix values are loaded before its
  // flag is awaited, so only x is on the dependency chain
  const int r = tid % BS, part = tid / BS;
  const int ndep = lower ? bi : nb - 1 - bi;
  const T *trow = Tp + (long)(r0 + r) * tr;
  T tv[16];
  auto load_t = [&](int d) {
    const int bj = lower ? d : nb - 1 - d, c0 = bj * BS, cols = min(BS, n - c0);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int c = part + 4 * m;
      tv[m] = (r < rows && c < cols) ? trow[(long)(c0 + c) * tc] : T(0);
    }
  };
  T acc[NR];
#pragma unroll
  for (int q = 0; q < NR; q++) acc[q] = T(0);
  if (ndep > 0) load_t(0);
  for (int d = 0; d < ndep; d++) {
    const int bj = lower ? d : nb - 1 - d, c0 = bj * BS, cols = min(BS, n - c0);
    if (lane == 0) {
      const uint64_t t0 = gtimer();
      while (ld_acquire(flags + bj) != epoch) {
        if (gtimer() - t0 > 1000000000ull) { atomicExch(err, 1); break; }
      }
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int c = part + 4 * m;
      if (c < cols) {
#pragma unroll
        for (int q = 0; q < NR; q++)
          if (q < nrhs) acc[q] = fma(tv[m], __ldcg(X + c0 + c + (long)q * ldx), acc[q]);
      }
    }
    if (d + 1 < ndep) load_t(d + 1);
  }
#pragma unroll
  for (int q = 0; q < NR; q++) sacc[part][r][q] = acc[q];
  __syncthreads();
  for (int idx = tid; idx < BS * NR; idx += 256) {
    const int rr = idx % BS, q = idx / BS;
    sx[rr][q] = sb[rr][q] - (sacc[0][rr][q] + sacc[1][rr][q] + sacc[2][rr][q] + sacc[3][rr][q]);
  }
  __syncthreads();
  // x = W (b - acc): thread (r, part) sums columns part*16 .. +15 of row r
  // (four short chains instead of one 64-long one), then the parts add up
#pragma unroll
  for (int q = 0; q < NR; q++) {
    T v = T(0);
#pragma unroll
    for (int c = 16 * part; c < 16 * part + 16; c++) v = fma(sW[r][c], sx[c][q], v);
    sacc[part][r][q] = v;
  }
  __syncthreads();
  for (int idx = tid; idx < BS * NR; idx += 256) {
    const int rr = idx % BS, q = idx / BS;
    if (rr >= rows || q >= nrhs) continue;
    X[r0 + rr + (long)q * ldx] = (sacc[0][rr][q] + sacc[1][rr][q]) + (sacc[2][rr][q] + sacc[3][rr][q]);
  }
  __syncthreads();
  if (tid == 0) {  // the barrier orders every thread's x stores before this release
    __threadfence();
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + bi), "r"(epoch) : "memory");
  }
}

}  // namespace

// Inverted 64x64 diagonal blocks of op(A)'s triangle, as trsv_w_dev takes them.
template <typename T>
void trsv_inverse_dev(int uplo, int trans, int diag, int n, const T *A, long lda, T *W, cudaStream_t st) {
  if (n <= 0) return;
  const bool tr = trans != kNoTrans;
  const long tstr = tr ? lda : 1, tcol = tr ? 1 : lda;
  const int lower = (uplo == kLower) != tr;
  trinv_dev<T>(n, A, tstr, tcol, lower, diag == kUnit, W, st);
}
template void trsv_inverse_dev<double>(int, int, int, int, const double *, long, double *, cudaStream_t);
template void trsv_inverse_dev<float>(int, int, int, int, const float *, long, float *, cudaStream_t);

// Solve op(A) X = B in place for nrhs <= 8 right-hand sides (Left side only).
template <typename T>
void trsv_dev(int uplo, int trans, int diag, int n, int nrhs, const T *A, long lda, T *B, long ldb,
              cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return;
  T *W = (T *)scratch(kSlotTrsmW, sizeof(T) * (size_t)cdiv(n, BS) * BS * BS);
  trsv_inverse_dev<T>(uplo, trans, diag, n, A, lda, W, st);
  trsv_w_dev<T>(uplo, trans, n, nrhs, A, lda, W, B, ldb, st);
}
template void trsv_dev<double>(int, int, int, int, int, const double *, long, double *, long, cudaStream_t);
template void trsv_dev<float>(int, int, int, int, int, const float *, long, float *, long, cudaStream_t);

// The same solve with the inverted diagonal blocks W already computed
// (trsv_inverse_dev): for repeated solves with one factor.
template <typename T>
void trsv_w_dev(int uplo, int trans, int n, int nrhs, const T *A, long lda, const T *W, T *B, long ldb,
                cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return;
  const bool tr = trans != kNoTrans;
  const long tstr = tr ? lda : 1, tcol = tr ? 1 : lda;  // effective T(i,k) = A[i*tstr + k*tcol]
  const int lower = (uplo == kLower) != tr;
  const int nb = cdiv(n, BS);
  // workspace: ticket counter, error word, flags
  int *ctl = (int *)scratch(kSlotTrsvCtl, sizeof(int) * (nb + 64));
  const int epoch = 1;
  int *counter = ctl, *err = ctl + 1, *flags = ctl + 64;
  ATLB_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(int) * (nb + 64), st));  // counter, flags
  constexpr int smem = BS * (BS + 1) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  if (nrhs == 1) trsv_kernel<T, 1><<<nb, 256, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  else if (nrhs <= 4) trsv_kernel<T, 4><<<nb, 256, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  else trsv_kernel<T, 8><<<nb, 256, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trsv_w_dev<double>(int, int, int, int, const double *, long, const double *, double *, long,
                                 cudaStream_t);
template void trsv_w_dev<float>(int, int, int, int, const float *, long, const float *, float *, long,
                                cudaStream_t);

}  // namespace atlb
