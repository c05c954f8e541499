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
#include <vector>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int CLEAF = 64;

// Factor the n x n (n <= 64) diagonal block at A in place; first
// non-positive pivot j lowers *dinfo to ioff + j + 1 and stops the block.
// Thread (i, g) keeps row i's columns g, g+4, ... of L in registers (the
// upper case works on the transpose, U = L^T).  Each step needs column j of
// the partially updated matrix; its owners publish it to a double-buffered
// shared copy at the end of the previous step, so a step costs one barrier.
template <typename T>
__global__ void __launch_bounds__(256)
potf2_kernel(int n, T *A, long lda, int upper, int *dinfo, int ioff) {
  static_assert(CLEAF == 64, "4 threads per row, 16 columns each");
  __shared__ T pcol[2][CLEAF];
  const int tid = threadIdx.x, i = tid % CLEAF, g = tid / CLEAF;
  T a[CLEAF / 4];
#pragma unroll
  for (int m = 0; m < CLEAF / 4; m++) {
    const int k = g + 4 * m;
    a[m] = (i < n && k <= i) ? (upper ? A[k + (long)i * lda] : A[i + (long)k * lda]) : T(0);
  }
  if (g == 0) pcol[0][i] = a[0];
  __syncthreads();
#pragma unroll 1
  for (int j = 0; j < n; j++) {
    const int b = j & 1;
    const T djj = pcol[b][j];
    if (!(djj > T(0))) {
      if (tid == 0) atomicMin(dinfo, ioff + j + 1);
      break;  // uniform: every thread read the same pivot
    }
    const T d = sqrt(djj), rd = T(1) / d;
    if (i >= j && i < n) {
      const T li = i == j ? d : pcol[b][i] * rd;
#pragma unroll
      for (int m = 0; m < CLEAF / 4; m++) {
        const int k = g + 4 * m;
        if (k == j) a[m] = li;
        else if (k > j && k <= i) a[m] = fma(-li, pcol[b][k] * rd, a[m]);
      }
    }
    if (g == ((j + 1) & 3) && i > j && i < n) {
      T v = T(0);
#pragma unroll
      for (int m = 0; m < CLEAF / 4; m++)
        if (g + 4 * m == j + 1) v = a[m];
      pcol[b ^ 1][i] = v;
    }
    __syncthreads();
  }
  if (i < n) {
#pragma unroll
    for (int m = 0; m < CLEAF / 4; m++) {
      const int k = g + 4 * m;
      if (k <= i) {
        if (upper) A[k + (long)i * lda] = a[m];
        else A[i + (long)k * lda] = a[m];
      }
    }
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

// C -= op(X) op(Y), everything with leading dimension lda
void offdiag_update(SgemmFn, int ta, int tb, int m, int n, int k, const double *X, const double *Y,
                    double *C, long lda, cudaStream_t st) {
  dgemm_dev(ta, tb, m, n, k, -1.0, X, lda, Y, lda, 1.0, C, lda, st);
}
void offdiag_update(SgemmFn fn, int ta, int tb, int m, int n, int k, const float *X, const float *Y,
                    float *C, long lda, cudaStream_t st) {
  (fn ? fn : sgemm_dev)(ta, tb, m, n, k, -1.f, X, lda, Y, lda, 1.f, C, lda, st, 0);
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

template <typename T>
void potrf_dev(int uplo, int N, T *A, long lda, int *dinfo, cudaStream_t st, SgemmFn gemm) {
  const int NBO = tune(kTunePotrfNB);  // multiple of 64
  const std::vector<unsigned long long> key = {21ull + sizeof(T), (unsigned long long)tune_generation(),
      (unsigned long long)uplo,
      (unsigned long long)N, (unsigned long long)lda, (unsigned long long)(uintptr_t)A,
      (unsigned long long)(uintptr_t)dinfo, (unsigned long long)(uintptr_t)gemm,
      (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    set_info_kernel_launch(dinfo, st);
    const bool up = uplo == kUpper;
    const int nblk = cdiv(N, NBO);
    if (nblk <= 1 || !lookahead_enabled()) {
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
    } else {
      // Look-ahead of depth one (as in getrf): after the main stream's TRSM
      // of block column k, the side stream updates and factors diagonal
      // block k+1 while the main stream updates the rest of the trailing
      // matrix (disjoint writes).
      cudaStream_t s1 = side_stream();
      potrf_rec<T>(up, 0, std::min(NBO, N), A, lda, dinfo, st, gemm);
      for (int k = 0; k < nblk - 1; k++) {
        const int j = k * NBO, jb = std::min(NBO, N - j), jn = j + jb, nr = N - jn;
        const int jbn = std::min(NBO, nr), nrest = nr - jbn;
        T *Ad = A + j + (long)j * lda, *Dn = A + jn + (long)jn * lda;
        if (k > 0) ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + (k & 1)), 0));  // block k factored
        T *P;  // the TRSM'd block column (lower) / block row (upper) of block k
        if (!up) {
          P = Ad + jb;
          trsm_dev<T>(kRight, kLower, kTrans, kNonUnit, nr, jb, T(1), Ad, lda, P, lda, st, gemm);
        } else {
          P = Ad + (long)jb * lda;
          trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, jb, nr, T(1), Ad, lda, P, lda, st, gemm);
        }
        ATLB_CUDA_CHECK(cudaEventRecord(side_event(k & 1), st));
        ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(k & 1), 0));
        {
          SideScope side;
          syrk_update(gemm, up, jbn, jb, P, Dn, lda, s1);   // diagonal block k+1
          potrf_rec<T>(up, jn, jbn, A, lda, dinfo, s1, gemm);
          ATLB_CUDA_CHECK(cudaEventRecord(side_event(2 + ((k + 1) & 1)), s1));
        }
        if (nrest > 0) {
          if (!up) {
            const T *Pn = P, *Pr = P + jbn;          // rows of block k+1 / below it
            offdiag_update(gemm, kNoTrans, kTrans, nrest, jbn, jb, Pr, Pn, Dn + jbn, lda, st);
            syrk_update(gemm, 0, nrest, jb, Pr, Dn + jbn + (long)jbn * lda, lda, st);
          } else {
            const T *Pn = P, *Pr = P + (long)jbn * lda;  // columns of block k+1 / right of it
            offdiag_update(gemm, kTrans, kNoTrans, jbn, nrest, jb, Pn, Pr, Dn + (long)jbn * lda, lda, st);
            syrk_update(gemm, 1, nrest, jb, Pr, Dn + jbn + (long)jbn * lda, lda, st);
          }
        }
      }
      ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + ((nblk - 1) & 1)), 0));  // join
    }
    finish_info_kernel_launch(dinfo, st);
  });
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
