// Cholesky factorization (clapack_dpotrf / ATL_potrfL, ATL_potrfU) and solve
// (ATL_potrs).
//
// Driver: the reference's recursion (src/lapack/ATL_potrfL.c:204-263,
// ATL_potrfU.c:199-257): factor the leading half, TRSM the off-diagonal block
// against it, SYRK-update the trailing half (the DMMA GEMM restricted to one
// triangle), factor the trailing half.  Leaves of <= 64 columns are factored
// by one CTA in shared memory; the upper case is factored as the transpose
// of the lower one (U = L^T), so a single leaf kernel serves both.
#include <algorithm>
#include <cmath>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int CLEAF = 64;

// Factor the n x n (n <= 64) diagonal block at A in place; first
// non-positive pivot j lowers *dinfo to ioff + j + 1 and stops the block.
template <typename T>
__global__ void __launch_bounds__(256)
potf2_kernel(int n, T *A, long lda, int upper, int *dinfo, int ioff) {
  __shared__ T s[CLEAF][CLEAF + 1];
  __shared__ int fail;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    int i = idx % n, k = idx / n;  // element (i, k) of the stored block
    T v = A[i + (long)k * lda];
    if (!upper) s[i][k] = v; else s[k][i] = v;  // work on L (lower)
  }
  if (tid == 0) fail = 0;
  __syncthreads();
  for (int j = 0; j < n; j++) {
    T d = s[j][j];
    if (!(d > T(0))) {
      if (tid == 0) { atomicMin(dinfo, ioff + j + 1); fail = 1; }
      break;
    }
    d = sqrt(d);
    __syncthreads();
    if (tid == 0) s[j][j] = d;
    for (int i = j + 1 + tid; i < n; i += blockDim.x) s[i][j] /= d;
    __syncthreads();
    const int m = n - j - 1;
    for (int idx = tid; idx < m * m; idx += blockDim.x) {
      int i = j + 1 + idx % m, k = j + 1 + idx / m;
      if (k <= i) s[i][k] -= s[i][j] * s[k][j];
    }
    __syncthreads();
  }
  __syncthreads();
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    int i = idx % n, k = idx / n;
    if (!upper) { if (i >= k) A[i + (long)k * lda] = s[i][k]; }
    else { if (i <= k) A[i + (long)k * lda] = s[k][i]; }
  }
}

void syrk_update(SgemmFn, int upper, int n, int k, const double *X, double *C, long lda,
                 cudaStream_t st) {
  if (!upper) dgemm_dev(kNoTrans, kTrans, n, n, k, -1.0, X, lda, X, lda, 1.0, C, lda, st, 1);
  else dgemm_dev(kTrans, kNoTrans, n, n, k, -1.0, X, lda, X, lda, 1.0, C, lda, st, 2);
}
void syrk_update(SgemmFn fn, int upper, int n, int k, const float *X, float *C, long lda,
                 cudaStream_t st) {
  SgemmFn g = fn ? fn : sgemm_dev;
  if (!upper) g(kNoTrans, kTrans, n, n, k, -1.f, X, lda, X, lda, 1.f, C, lda, st, 1);
  else g(kTrans, kNoTrans, n, n, k, -1.f, X, lda, X, lda, 1.f, C, lda, st, 2);
}

template <typename T>
void potrf_rec(int upper, int off, int N, T *A, long lda, int *dinfo, cudaStream_t st,
               SgemmFn gemm) {
  if (N <= 0) return;
  T *Ad = A + off + (long)off * lda;
  if (N <= CLEAF) {
    potf2_kernel<T><<<1, 256, 0, st>>>(N, Ad, lda, upper, dinfo, off);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  const int Nl = std::max(CLEAF, (N / 2) / CLEAF * CLEAF), Nr = N - Nl;
  potrf_rec<T>(upper, off, Nl, A, lda, dinfo, st, gemm);
  if (!upper) {
    T *A21 = Ad + Nl, *A22 = Ad + Nl + (long)Nl * lda;
    trsm_dev<T>(kRight, kLower, kTrans, kNonUnit, Nr, Nl, T(1), Ad, lda, A21, lda, st, gemm);
    syrk_update(gemm, 0, Nr, Nl, A21, A22, lda, st);
  } else {
    T *A12 = Ad + (long)Nl * lda, *A22 = Ad + Nl + (long)Nl * lda;
    trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, Nl, Nr, T(1), Ad, lda, A12, lda, st, gemm);
    syrk_update(gemm, 1, Nr, Nl, A12, A22, lda, st);
  }
  potrf_rec<T>(upper, off + Nl, Nr, A, lda, dinfo, st, gemm);
}

}  // namespace

// Outer loop: NBO-wide diagonal blocks factored by the recursion above, then
// one TRSM for the block column below (right of) the diagonal block and one
// SYRK for the trailing matrix.
constexpr int NBO = 256;

template <typename T>
void potrf_dev(int uplo, int N, T *A, long lda, int *dinfo, cudaStream_t st, SgemmFn gemm) {
  set_info_kernel_launch(dinfo, st);
  const bool up = uplo == kUpper;
  for (int j = 0; j < N; j += NBO) {
    const int jb = std::min(NBO, N - j), nr = N - j - jb;
    T *Ad = A + j + (long)j * lda;
    potrf_rec<T>(up, j, jb, A, lda, dinfo, st, gemm);
    if (nr <= 0) break;
    if (!up) {
      T *A21 = Ad + jb, *A22 = Ad + jb + (long)jb * lda;
      trsm_dev<T>(kRight, kLower, kTrans, kNonUnit, nr, jb, T(1), Ad, lda, A21, lda, st, gemm);
      syrk_update(gemm, 0, nr, jb, A21, A22, lda, st);
    } else {
      T *A12 = Ad + (long)jb * lda, *A22 = Ad + jb + (long)jb * lda;
      trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, jb, nr, T(1), Ad, lda, A12, lda, st, gemm);
      syrk_update(gemm, 1, nr, jb, A12, A22, lda, st);
    }
  }
  finish_info_kernel_launch(dinfo, st);
}
template void potrf_dev<double>(int, int, double *, long, int *, cudaStream_t, SgemmFn);
template void potrf_dev<float>(int, int, float *, long, int *, cudaStream_t, SgemmFn);

template <typename T>
void potrs_dev(int uplo, int N, int NRHS, const T *A, long lda, T *B, long ldb, cudaStream_t st,
               SgemmFn gemm) {
  // ATL_potrs column-major (src/lapack/ATL_potrs.c:41-60)
  if (N <= 0 || NRHS <= 0) return;
  if (NRHS <= 8) {  // few right-hand sides: one-launch blocked solves
    if (uplo == kUpper) {
      trsv_dev<T>(kUpper, kTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
      trsv_dev<T>(kUpper, kNoTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
    } else {
      trsv_dev<T>(kLower, kNoTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
      trsv_dev<T>(kLower, kTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
    }
    return;
  }
  if (uplo == kUpper) {
    trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
    trsm_dev<T>(kLeft, kUpper, kNoTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
  } else {
    trsm_dev<T>(kLeft, kLower, kNoTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
    trsm_dev<T>(kLeft, kLower, kTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
  }
}
template void potrs_dev<double>(int, int, int, const double *, long, double *, long,
                                cudaStream_t, SgemmFn);
template void potrs_dev<float>(int, int, int, const float *, long, float *, long, cudaStream_t,
                               SgemmFn);

}  // namespace atlb
