// Cholesky factorization (clapack_dpotrf / ATL_potrfL, ATL_potrfU) and solve
// (ATL_potrs).
//
// Driver: the reference's recursion (src/lapack/ATL_potrfL.c:204-263,
// ATL_potrfU.c:199-257): factor the leading half, TRSM the off-diagonal block
// against it, SYRK-update the trailing half (the DMMA GEMM restricted to one
// triangle), factor the trailing half.  Leaves of <= 128 columns are factored
// by one CTA in shared memory (blocked: 16-column panels and register-tiled
// updates of the trailing triangle); the upper case is factored as the
// transpose of the lower one (U = L^T), so a single leaf kernel serves both.
#include <algorithm>
#include <cmath>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "chol_blocks.cuh"

namespace atlb {
namespace {

constexpr int CLEAF = 128;

// Factor the n x n (n <= 128) diagonal block at A in place in shared memory
// (cholb::chol_smem: 16-column panels, the trailing triangle updated on the
// FP64 tensor cores for double, with 4 x 4 register tiles for float); the
// upper case is loaded transposed (U = L^T).  A first non-positive pivot j lowers *dinfo to ioff + j + 1; the
// block is then left partly factored.
template <typename T>
__global__ void __launch_bounds__(256)
potrf_leaf_kernel(int n, T *A, long lda, int upper, int *dinfo, int ioff) {
  extern __shared__ __align__(16) unsigned char leaf_smem[];
  T *S = reinterpret_cast<T *>(leaf_smem);
  const int lds = cholb::ld_for(n);
  const int nn = n * n, tid = threadIdx.x;
  for (int base = 0; base < nn; base += 256 * 8) {  // eight loads in flight per thread
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, i = idx % n, k = idx / n;
      v[u] = (idx < nn && i >= k) ? (upper ? A[k + (long)i * lda] : A[i + (long)k * lda]) : T(0);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, i = idx % n, k = idx / n;
      if (idx < nn && i >= k) S[i + k * lds] = v[u];
    }
  }
  __syncthreads();
  const int fail = cholb::chol_smem(S, lds, n);
  if (fail && threadIdx.x == 0) atomicMin(dinfo, ioff + fail);
  for (int idx = tid; idx < nn; idx += 256) {
    const int i = idx % n, k = idx / n;
    if (i < k) continue;
    if (upper) A[k + (long)i * lda] = S[i + k * lds];
    else A[i + (long)k * lda] = S[i + k * lds];
  }
}

template <typename T>
void potrf_leaf(int n, T *Ad, long lda, int upper, int *dinfo, int ioff, cudaStream_t st) {
  const size_t smem = sizeof(T) * (size_t)n * cholb::ld_for(n);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(potrf_leaf_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(T) * CLEAF * cholb::ld_for(CLEAF))));
    configured = true;
  }
  potrf_leaf_kernel<T><<<1, 256, smem, st>>>(n, Ad, lda, upper, dinfo, ioff);
  ATLB_CUDA_CHECK(cudaGetLastError());
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
    potrf_leaf<T>(N, Ad, lda, upper, dinfo, off, st);
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
      // Look-ahead of depth one.  The side stream owns the chain of diagonal
      // blocks: once the main stream's wide update by block column k-1 is in
      // (it covers diagonal block k+1), the side stream updates diagonal
      // block k+1 by block column k, factors it, and -- once the main stream
      // has updated block column k+1 below the diagonal by block column k --
      // solves that block column (TRSM).  The main stream does that narrow
      // update first, then the wide update of the rest of the trailing
      // matrix, which overlaps the side stream's chain, so the TRSM is off
      // the main stream.  Writes never overlap: diagonal block k+1 and block
      // column k+1 below it (side), the trailing matrix beyond block column
      // k+1 (main), block column k+1 below the diagonal (main's narrow
      // update, ordered before the side's TRSM by an event).  Events:
      // 0/1 narrow update k done, 2/3 block column k solved, 4/5 wide
      // update k done.
      cudaStream_t s1 = side_stream();
      auto blk = [&](int k) { return A + (long)k * NBO + (long)k * NBO * lda; };  // diagonal block k
      auto trsm_col = [&](int k, cudaStream_t s) {  // block column k below its diagonal block
        const int j = k * NBO, jb = std::min(NBO, N - j), nr = N - j - jb;
        if (nr <= 0) return;
        T *Ad = blk(k);
        if (!up) trsm_dev<T>(kRight, kLower, kTrans, kNonUnit, nr, jb, T(1), Ad, lda, Ad + jb, lda, s, gemm);
        else trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, jb, nr, T(1), Ad, lda, Ad + (long)jb * lda, lda, s, gemm);
      };
      potrf_rec<T>(up, 0, std::min(NBO, N), A, lda, dinfo, st, gemm);
      trsm_col(0, st);
      ATLB_CUDA_CHECK(cudaEventRecord(side_event(0), st));
      ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(0), 0));  // block column 0 solved
      for (int k = 0; k < nblk - 1; k++) {
        const int j = k * NBO, jb = std::min(NBO, N - j), jn = j + jb, nr = N - jn;
        const int jbn = std::min(NBO, nr), nrest = nr - jbn;
        T *Ad = blk(k), *Dn = A + jn + (long)jn * lda;
        const T *P = up ? Ad + (long)jb * lda : Ad + jb;  // block column (row) k, solved
        if (k > 0) ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + (k & 1)), 0));  // block column k solved
        if (nrest > 0) {  // narrow update: block column k+1 below its diagonal block
          if (!up) offdiag_update(gemm, kNoTrans, kTrans, nrest, jbn, jb, P + jbn, P, Dn + jbn, lda, st);
          else offdiag_update(gemm, kTrans, kNoTrans, jbn, nrest, jb, P, P + (long)jbn * lda, Dn + (long)jbn * lda, lda, st);
        }
        ATLB_CUDA_CHECK(cudaEventRecord(side_event(k & 1), st));
        {
          SideScope side;
          if (k > 0) ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(4 + ((k - 1) & 1)), 0));  // wide update k-1 in
          syrk_update(gemm, up, jbn, jb, P, Dn, lda, s1);   // diagonal block k+1
          potrf_rec<T>(up, jn, jbn, A, lda, dinfo, s1, gemm);
          ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(k & 1), 0));  // its block column updated
          trsm_col(k + 1, s1);
          ATLB_CUDA_CHECK(cudaEventRecord(side_event(2 + ((k + 1) & 1)), s1));
        }
        if (nrest > 0) {  // wide update: the trailing matrix beyond block column k+1
          if (!up) syrk_update(gemm, 0, nrest, jb, P + jbn, Dn + jbn + (long)jbn * lda, lda, st);
          else syrk_update(gemm, 1, nrest, jb, P + (long)jbn * lda, Dn + jbn + (long)jbn * lda, lda, st);
        }
        ATLB_CUDA_CHECK(cudaEventRecord(side_event(4 + (k & 1)), st));
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
  if (NRHS <= kTrsvMaxRhs) {  // few right-hand sides: blocked solves, one launch per 8 columns
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
