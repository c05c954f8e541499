// Drop-in C entry points (cblas_* / clapack_* / ATL_dgeqrf) and the
// device-pointer extensions.  Argument checks mirror the reference's
// interface layer (interfaces/blas/C/src/cblas_*.c, interfaces/lapack/C/src/
// clapack_*.c): same positions, first bad argument reported.  Row-major calls
// are mapped onto the column-major device routines exactly as the reference
// maps them (operand swap for GEMM, side/uplo flips for TRSM/SYRK, the
// transposed factorization for getrf/getrs/potrf/potrs, LQ-of-the-view for
// geqrf).
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "mixed.h"
#include "../../include/atlas_b200.h"
#include "staging.h"

namespace atlb {
void xerbla(int pos, const char *rout);

namespace {

void sync(cudaStream_t st) { ATLB_CUDA_CHECK(cudaStreamSynchronize(st)); }

__global__ void reflect_upper_kernel(int n, double *C, long ldc) {
  long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    if (i > j) C[i + (long)j * ldc] = C[j + (long)i * ldc];
  }
}

}  // namespace

__global__ void transpose_kernel(int rows, int cols, const double *S, long lds, double *D,
                                 long ldd) {
  __shared__ double t[32][33];
  int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int r = bx + threadIdx.x, c = by + k;
    if (r < rows && c < cols) t[k][threadIdx.x] = S[r + (long)c * lds];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int r = by + threadIdx.x, c = bx + k;  // D is cols x rows
    if (r < cols && c < rows) D[r + (long)c * ldd] = t[threadIdx.x][k];
  }
}
void transpose_dev(int rows, int cols, const double *S, long lds, double *D, long ldd,
                   cudaStream_t st) {
  dim3 grid(cdiv(rows, 32), cdiv(cols, 32)), block(32, 8);
  transpose_kernel<<<grid, block, 0, st>>>(rows, cols, S, lds, D, ldd);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

namespace {

inline bool bad_trans(int t) { return t != kNoTrans && t != kTrans && t != kConjTrans; }

// col-major GEMM on device with the reference's A==B SYRK shortcut
// (interfaces/blas/C/src/cblas_dgemm.c:123-129)
void dgemm_core(int ta, int tb, int M, int N, int K, double alpha, const double *A, long lda,
                const double *B, long ldb, double beta, double *C, long ldc, cudaStream_t st,
                bool syrk_shortcut) {
  if (syrk_shortcut) {
    dgemm_dev(ta, tb, N, N, K, alpha, A, lda, B, ldb, 0.0, C, ldc, st, 2);
    long total = (long)N * N;
    reflect_upper_kernel<<<(int)std::min<long>((total + 255) / 256, 4096), 256, 0, st>>>(N, C, ldc);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  dgemm_dev(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, 0);
}

}  // namespace
}  // namespace atlb

using namespace atlb;

extern "C" {

// ---------------------------------------------------------------- BLAS

void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_TRANSPOSE TB, const int M, const int N, const int K,
                 const double alpha, const double *A, const int lda, const double *B,
                 const int ldb, const double beta, double *C, const int ldc) {
  int info = 2000;
  auto e = [&](int p) { info = std::min(info, p); };
  if (M < 0) e(4);
  if (N < 0) e(5);
  if (K < 0) e(6);
  if (Order == CblasRowMajor) {
    if (TA == CblasNoTrans) { if (lda < K || lda < 1) e(9); }
    else { if (bad_trans(TA)) e(2); if (lda < M || lda < 1) e(9); }
    if (TB == CblasNoTrans) { if (ldb < N || ldb < 1) e(11); }
    else { if (bad_trans(TB)) e(3); if (ldb < K || ldb < 1) e(11); }
    if (ldc < N || ldc < 1) e(14);
  } else if (Order == CblasColMajor) {
    if (TA == CblasNoTrans) { if (lda < M || lda < 1) e(9); }
    else { if (bad_trans(TA)) e(2); if (lda < K || lda < 1) e(9); }
    if (TB == CblasNoTrans) { if (ldb < K || ldb < 1) e(11); }
    else { if (bad_trans(TB)) e(3); if (ldb < N || ldb < 1) e(11); }
    if (ldc < M || ldc < 1) e(14);
  } else e(1);
  if (info != 2000) { xerbla(info, "cblas_dgemm"); return; }
  if (M == 0 || N == 0) return;
  cudaStream_t st = stream();
  // column-major problem: C(m x n) = op(a) op(b)
  const bool col = Order == CblasColMajor;
  int ta = col ? TA : TB, tb = col ? TB : TA, m = col ? M : N, n = col ? N : M;
  const double *a = col ? A : B, *b = col ? B : A;
  long la = col ? lda : ldb, lb = col ? ldb : lda;
  const bool shortcut = (A == B && M == N && TA != TB && lda == ldb && beta == 0.0);
  if (shortcut) { ta = col ? TA : TB; tb = (ta == CblasNoTrans) ? CblasTrans : CblasNoTrans; }
  DMat<double> dA = stage_in(kSlotA, a, ta == kNoTrans ? m : K, ta == kNoTrans ? K : m, la, true, st);
  DMat<double> dB = shortcut ? dA
                             : stage_in(kSlotB, b, tb == kNoTrans ? K : n, tb == kNoTrans ? n : K, lb, true, st);
  DMat<double> dC = stage_in(kSlotC, C, m, n, ldc, beta != 0.0, st);
  dgemm_core(ta, tb, m, n, K, alpha, dA.d, dA.ld, dB.d, dB.ld, beta, dC.d, dC.ld, st, shortcut);
  stage_out(C, ldc, dC, m, n, st);
  sync(st);
}

void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_TRANSPOSE TB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc) {
  int info = 2000;
  auto e = [&](int p) { info = std::min(info, p); };
  if (M < 0) e(4);
  if (N < 0) e(5);
  if (K < 0) e(6);
  if (Order == CblasRowMajor) {
    if (TA == CblasNoTrans) { if (lda < K || lda < 1) e(9); }
    else { if (bad_trans(TA)) e(2); if (lda < M || lda < 1) e(9); }
    if (TB == CblasNoTrans) { if (ldb < N || ldb < 1) e(11); }
    else { if (bad_trans(TB)) e(3); if (ldb < K || ldb < 1) e(11); }
    if (ldc < N || ldc < 1) e(14);
  } else if (Order == CblasColMajor) {
    if (TA == CblasNoTrans) { if (lda < M || lda < 1) e(9); }
    else { if (bad_trans(TA)) e(2); if (lda < K || lda < 1) e(9); }
    if (TB == CblasNoTrans) { if (ldb < K || ldb < 1) e(11); }
    else { if (bad_trans(TB)) e(3); if (ldb < N || ldb < 1) e(11); }
    if (ldc < M || ldc < 1) e(14);
  } else e(1);
  if (info != 2000) { xerbla(info, "cblas_sgemm"); return; }
  if (M == 0 || N == 0) return;
  cudaStream_t st = stream();
  const bool col = Order == CblasColMajor;
  int ta = col ? TA : TB, tb = col ? TB : TA, m = col ? M : N, n = col ? N : M;
  const float *a = col ? A : B, *b = col ? B : A;
  long la = col ? lda : ldb, lb = col ? ldb : lda;
  DMat<float> dA = stage_in(kSlotA, a, ta == kNoTrans ? m : K, ta == kNoTrans ? K : m, la, true, st);
  DMat<float> dB = stage_in(kSlotB, b, tb == kNoTrans ? K : n, tb == kNoTrans ? n : K, lb, true, st);
  DMat<float> dC = stage_in(kSlotC, C, m, n, ldc, beta != 0.f, st);
  sgemm_dev(ta, tb, m, n, K, alpha, dA.d, dA.ld, dB.d, dB.ld, beta, dC.d, dC.ld, st, 0);
  stage_out(C, ldc, dC, m, n, st);
  sync(st);
}

static int trsm_like_checks(const char *name, int Order, int Side, int Uplo, int TA, int Diag,
                            int M, int N, int lda, int ldb) {
  // interfaces/blas/C/src/cblas_dtrsm.c:20-90 (cblas_dtrmm.c has the same)
  int info = 2000;
  auto e = [&](int p) { info = std::min(info, p); };
  if (Order == CblasColMajor || Order == CblasRowMajor) {
    if (Side == CblasLeft) { if (lda < M || lda < 1) e(10); }
    else if (Side == CblasRight) { if (lda < N || lda < 1) e(10); }
    else e(2);
    if (Order == CblasColMajor) { if (ldb < M || ldb < 1) e(12); }
    else { if (ldb < N || ldb < 1) e(12); }
  } else e(1);
  if (Uplo != CblasUpper && Uplo != CblasLower) e(3);
  if (bad_trans(TA)) e(4);
  if (Diag != CblasUnit && Diag != CblasNonUnit) e(5);
  if (M < 0) e(6);
  if (N < 0) e(7);
  if (info != 2000) { xerbla(info, name); return info; }
  return 0;
}

void cblas_dtrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb) {
  if (trsm_like_checks("cblas_dtrsm", Order, Side, Uplo, TA, Diag, M, N, lda, ldb)) return;
  if (M == 0 || N == 0) return;
  cudaStream_t st = stream();
  int side = Side, uplo = Uplo, m = M, n = N;
  if (Order == CblasRowMajor) {
    side = (Side == CblasLeft) ? kRight : kLeft;
    uplo = (Uplo == CblasUpper) ? kLower : kUpper;
    m = N; n = M;
  }
  int na = side == kLeft ? m : n;
  DMat<double> dA = stage_in(kSlotA, A, na, na, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, m, n, ldb, alpha != 0.0, st);
  trsm_dev<double>(side, uplo, (int)TA == kNoTrans ? kNoTrans : kTrans, Diag, m, n, alpha, dA.d, dA.ld,
                   dB.d, dB.ld, st);
  stage_out(B, ldb, dB, m, n, st);
  sync(st);
}

void cblas_dtrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb) {
  if (trsm_like_checks("cblas_dtrmm", Order, Side, Uplo, TA, Diag, M, N, lda, ldb)) return;
  if (M == 0 || N == 0) return;
  cudaStream_t st = stream();
  int side = Side, uplo = Uplo, m = M, n = N;
  if (Order == CblasRowMajor) {
    side = (Side == CblasLeft) ? kRight : kLeft;
    uplo = (Uplo == CblasUpper) ? kLower : kUpper;
    m = N; n = M;
  }
  int na = side == kLeft ? m : n;
  DMat<double> dA = stage_in(kSlotA, A, na, na, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, m, n, ldb, true, st);
  dtrmm_dev(side, uplo, (int)TA == kNoTrans ? kNoTrans : kTrans, Diag, m, n, alpha, dA.d, dA.ld, dB.d,
            dB.ld, st);
  stage_out(B, ldb, dB, m, n, st);
  sync(st);
}

void cblas_dsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const double *A, const int lda, const double beta, double *C, const int ldc) {
  // interfaces/blas/C/src/cblas_dsyrk.c:20-75
  int info = 2000;
  auto e = [&](int p) { info = std::min(info, p); };
  if (Uplo != CblasUpper && Uplo != CblasLower) e(2);
  if (N < 0) e(4);
  if (K < 0) e(5);
  if (Order == CblasColMajor) {
    if (Trans == CblasNoTrans) { if (lda < N || lda < 1) e(8); }
    else { if (Trans != CblasTrans && Trans != CblasConjTrans) e(3); if (lda < K || lda < 1) e(8); }
  } else if (Order == CblasRowMajor) {
    if (Trans == CblasNoTrans) { if (lda < K || lda < 1) e(8); }
    else { if (Trans != CblasTrans && Trans != CblasConjTrans) e(3); if (lda < N || lda < 1) e(8); }
  } else e(1);
  if (ldc < N || ldc < 1) e(11);
  if (info != 2000) { xerbla(info, "cblas_dsyrk"); return; }
  if (N == 0) return;
  cudaStream_t st = stream();
  int uplo = Uplo, trans = (Trans == CblasNoTrans) ? kNoTrans : kTrans;
  if (Order == CblasRowMajor) {
    uplo = (Uplo == CblasUpper) ? kLower : kUpper;
    trans = (trans == kNoTrans) ? kTrans : kNoTrans;
  }
  int ar = trans == kNoTrans ? N : K, ac = trans == kNoTrans ? K : N;
  DMat<double> dA = stage_in(kSlotA, A, ar, ac, lda, true, st);
  DMat<double> dC = stage_in(kSlotC, C, N, N, ldc, true, st);
  int tri = (uplo == kLower) ? 1 : 2;
  if (trans == kNoTrans)
    dgemm_dev(kNoTrans, kTrans, N, N, K, alpha, dA.d, dA.ld, dA.d, dA.ld, beta, dC.d, dC.ld, st, tri);
  else
    dgemm_dev(kTrans, kNoTrans, N, N, K, alpha, dA.d, dA.ld, dA.d, dA.ld, beta, dC.d, dC.ld, st, tri);
  stage_out(C, ldc, dC, N, N, st);
  sync(st);
}

// ---------------------------------------------------------------- LAPACK

int clapack_dgetrf(const enum CBLAS_ORDER Order, const int M, const int N, double *A,
                   const int lda, int *ipiv) {
  // interfaces/lapack/C/src/clapack_dgetrf.c:49-86
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (M < 0) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (Order == CblasColMajor) { if (lda < M || lda < 1) { if (!ierr) ierr = -6; } }
  else { if (lda < N || lda < 1) { if (!ierr) ierr = -6; } }
  if (ierr) { xerbla(-ierr, "clapack_dgetrf"); return ierr; }
  // row-major A = L U P (unit U) is the column-major factorization of the
  // N x M transposed view (src/lapack/ATL_getrfR.c)
  const int m = Order == CblasColMajor ? M : N, n = Order == CblasColMajor ? N : M;
  const int mn = std::min(m, n);
  if (mn == 0) return 0;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, m, n, lda, true, st);
  int *dip = stage_vec_in<int>(kSlotIpiv, ipiv, mn, false, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  getrf_dev<double>(m, n, dA.d, dA.ld, dip, dinfo, st);
  stage_out(A, lda, dA, m, n, st);
  stage_vec_out<int>(ipiv, dip, mn, st);
  int *hinfo = (int *)pinned(kSlotInfo, 64);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  sync(st);
  return *hinfo;
}

int clapack_dgetrs(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE Trans, const int N,
                   const int NRHS, const double *A, const int lda, const int *ipiv, double *B,
                   const int ldb) {
  // interfaces/lapack/C/src/clapack_dgetrs.c:19-57
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (bad_trans(Trans)) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (NRHS < 0) { if (!ierr) ierr = -4; }
  if (lda < N || lda < 1) { if (!ierr) ierr = -6; }
  if (ldb < N || ldb < 1) { if (!ierr) ierr = -9; }
  if (ierr) { xerbla(-ierr, "clapack_dgetrs"); return ierr; }
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  // row-major: the stored factors are those of A^T, so the solve flips Trans
  int tr = (Trans == CblasNoTrans) ? kNoTrans : kTrans;
  if (Order == CblasRowMajor) tr = (tr == kNoTrans) ? kTrans : kNoTrans;
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  int *dip = stage_vec_in<int>(kSlotIpiv, ipiv, N, true, st);
  DMat<double> dB = stage_in(kSlotB, B, N, NRHS, ldb, true, st);
  getrs_dev<double>(tr, N, NRHS, dA.d, dA.ld, dip, dB.d, dB.ld, st);
  stage_out(B, ldb, dB, N, NRHS, st);
  sync(st);
  return 0;
}

int clapack_dgesv(const enum CBLAS_ORDER Order, const int N, const int NRHS, double *A,
                  const int lda, int *ipiv, double *B, const int ldb) {
  // interfaces/lapack/C/src/clapack_dgesv.c:19-62
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (N < 0) { if (!ierr) ierr = -2; }
  if (NRHS < 0) { if (!ierr) ierr = -3; }
  if (lda < N || lda < 1) { if (!ierr) ierr = -5; }
  if (ldb < N || ldb < 1) { if (!ierr) ierr = -8; }
  if (ierr) { xerbla(-ierr, "clapack_dgesv"); return ierr; }
  if (N == 0) return 0;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  int *dip = stage_vec_in<int>(kSlotIpiv, ipiv, N, false, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  getrf_dev<double>(N, N, dA.d, dA.ld, dip, dinfo, st);
  int *hinfo = (int *)pinned(kSlotInfo, 64);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  stage_out(A, lda, dA, N, N, st);
  stage_vec_out<int>(ipiv, dip, N, st);
  sync(st);
  int info = *hinfo;
  if (info == 0 && NRHS > 0) {
    int tr = Order == CblasColMajor ? kNoTrans : kTrans;
    DMat<double> dB = stage_in(kSlotB, B, N, NRHS, ldb, true, st);
    getrs_dev<double>(tr, N, NRHS, dA.d, dA.ld, dip, dB.d, dB.ld, st);
    stage_out(B, ldb, dB, N, NRHS, st);
    sync(st);
  }
  return info;
}

static int potrf_checks(const char *name, int Order, int Uplo, int N, int lda) {
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (Uplo != CblasUpper && Uplo != CblasLower) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (lda < N || lda < 1) { if (!ierr) ierr = -5; }
  if (ierr) xerbla(-ierr, name);
  return ierr;
}

int clapack_dpotrf(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                   double *A, const int lda) {
  // interfaces/lapack/C/src/clapack_dpotrf.c:19-43; row-major Upper is the
  // column-major Lower factorization of the same buffer (src/lapack/ATL_potrf.c:16-27)
  int ierr = potrf_checks("clapack_dpotrf", Order, Uplo, N, lda);
  if (ierr) return ierr;
  if (N == 0) return 0;
  cudaStream_t st = stream();
  int uplo = Uplo;
  if (Order == CblasRowMajor) uplo = (Uplo == CblasUpper) ? kLower : kUpper;
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  potrf_dev<double>(uplo, N, dA.d, dA.ld, dinfo, st);
  stage_out(A, lda, dA, N, N, st);
  int *hinfo = (int *)pinned(kSlotInfo, 64);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  sync(st);
  return *hinfo;
}

int clapack_dpotrs(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                   const int NRHS, const double *A, const int lda, double *B, const int ldb) {
  // interfaces/lapack/C/src/clapack_dpotrs.c:19-56
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (Uplo != CblasUpper && Uplo != CblasLower) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (NRHS < 0) { if (!ierr) ierr = -4; }
  if (lda < N || lda < 1) { if (!ierr) ierr = -6; }
  if (ldb < N || ldb < 1) { if (!ierr) ierr = -8; }
  if (ierr) { xerbla(-ierr, "clapack_dpotrs"); return ierr; }
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  int uplo = Uplo;
  if (Order == CblasRowMajor) uplo = (Uplo == CblasUpper) ? kLower : kUpper;
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, N, NRHS, ldb, true, st);
  potrs_dev<double>(uplo, N, NRHS, dA.d, dA.ld, dB.d, dB.ld, st);
  stage_out(B, ldb, dB, N, NRHS, st);
  sync(st);
  return 0;
}

int clapack_dposv(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                  const int NRHS, double *A, const int lda, double *B, const int ldb) {
  // interfaces/lapack/C/src/clapack_dposv.c:19-58
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (Uplo != CblasUpper && Uplo != CblasLower) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (NRHS < 0) { if (!ierr) ierr = -4; }
  if (lda < N || lda < 1) { if (!ierr) ierr = -6; }
  if (ldb < N || ldb < 1) { if (!ierr) ierr = -8; }
  if (ierr) { xerbla(-ierr, "clapack_dposv"); return ierr; }
  if (N == 0) return 0;
  cudaStream_t st = stream();
  int uplo = Uplo;
  if (Order == CblasRowMajor) uplo = (Uplo == CblasUpper) ? kLower : kUpper;
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  potrf_dev<double>(uplo, N, dA.d, dA.ld, dinfo, st);
  int *hinfo = (int *)pinned(kSlotInfo, 64);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  stage_out(A, lda, dA, N, N, st);
  sync(st);
  int info = *hinfo;
  if (info == 0 && NRHS > 0) {
    DMat<double> dB = stage_in(kSlotB, B, N, NRHS, ldb, true, st);
    potrs_dev<double>(uplo, N, NRHS, dA.d, dA.ld, dB.d, dB.ld, st);
    stage_out(B, ldb, dB, N, NRHS, st);
    sync(st);
  }
  return info;
}

static int geqrf_nb() { return 32; }

int ATL_dgeqrf(const int M, const int N, double *A, const int lda, double *TAU, double *WORK,
               const int LWORK) {
  // src/lapack/ATL_geqrf.c:117-143: LWORK < 0 is a workspace query
  const int nb = geqrf_nb();
  if (LWORK < 0) {
    if (WORK) *WORK = (double)(N * nb + nb * nb + std::max(M, N));
    return 0;
  }
  if (M < 1 || N < 1) return 0;
  cudaStream_t st = stream();
  const int mn = std::min(M, N);
  DMat<double> dA = stage_in(kSlotA, A, M, N, lda, true, st);
  double *dtau = stage_vec_in<double>(kSlotTau, TAU, mn, false, st);
  dgeqrf_dev(M, N, dA.d, dA.ld, dtau, st);
  stage_out(A, lda, dA, M, N, st);
  stage_vec_out<double>(TAU, dtau, mn, st);
  sync(st);
  return 0;
}

int clapack_dgeqrf(const enum CBLAS_ORDER Order, const int M, const int N, double *A,
                   const int lda, double *TAU) {
  // interfaces/lapack/C/src/clapack_dgeqrf.c:19-61
  int ierr = 0;
  if (Order != CblasRowMajor && Order != CblasColMajor) { if (!ierr) ierr = -1; }
  if (M < 0) { if (!ierr) ierr = -2; }
  if (N < 0) { if (!ierr) ierr = -3; }
  if (Order == CblasColMajor) { if (lda < M || lda < 1) { if (!ierr) ierr = -5; } }
  else { if (lda < N || lda < 1) { if (!ierr) ierr = -5; } }
  if (ierr) { xerbla(-ierr, "clapack_dgeqrf"); return ierr; }
  if (Order == CblasColMajor) return ATL_dgeqrf(M, N, A, lda, TAU, nullptr, 0);
  // Row-major: the reference computes the LQ factorization of the N x M
  // column-major view (ATL_dgelqf).  For real data that is the QR
  // factorization of the view's transpose -- the logical M x N row-major
  // matrix -- with the same reflectors and tau, stored transposed.
  if (M < 1 || N < 1) return 0;
  cudaStream_t st = stream();
  const int mn = std::min(M, N);
  DMat<double> dV = stage_in(kSlotA, A, N, M, lda, true, st);  // the col-major view, N x M
  double *T = (double *)scratch(kSlotC, sizeof(double) * (size_t)M * N);  // not kSlotWork: dgeqrf_dev uses it
  transpose_dev(N, M, dV.d, dV.ld, T, M, st);  // T = view^T, M x N
  double *dtau = stage_vec_in<double>(kSlotTau, TAU, mn, false, st);
  dgeqrf_dev(M, N, T, M, dtau, st);
  transpose_dev(M, N, T, M, dV.d, dV.ld, st);
  stage_out(A, lda, dV, N, M, st);
  stage_vec_out<double>(TAU, dtau, mn, st);
  sync(st);
  return 0;
}

// ---------------------------------------------------------------- device API

int atlb_dgemm_dev(int TA, int TB, int M, int N, int K, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc) {
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (bad_trans(TA)) return -1;
  if (bad_trans(TB)) return -2;
  if (lda < std::max(1, TA == kNoTrans ? M : K)) return -8;
  if (ldb < std::max(1, TB == kNoTrans ? K : N)) return -10;
  if (ldc < std::max(1, M)) return -13;
  dgemm_dev(TA == kNoTrans ? kNoTrans : kTrans, TB == kNoTrans ? kNoTrans : kTrans, M, N, K, alpha,
            A, lda, B, ldb, beta, C, ldc, stream(), 0);
  return 0;
}

int atlb_sgemm_dev(int TA, int TB, int M, int N, int K, float alpha, const float *A, int lda,
                   const float *B, int ldb, float beta, float *C, int ldc) {
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (bad_trans(TA)) return -1;
  if (bad_trans(TB)) return -2;
  if (lda < std::max(1, TA == kNoTrans ? M : K)) return -8;
  if (ldb < std::max(1, TB == kNoTrans ? K : N)) return -10;
  if (ldc < std::max(1, M)) return -13;
  sgemm_dev(TA == kNoTrans ? kNoTrans : kTrans, TB == kNoTrans ? kNoTrans : kTrans, M, N, K, alpha,
            A, lda, B, ldb, beta, C, ldc, stream(), 0);
  return 0;
}

int atlb_sgemm_tc_dev(int prec, int TA, int TB, int M, int N, int K, float alpha, const float *A,
                      int lda, const float *B, int ldb, float beta, float *C, int ldc) {
  if (prec != 1 && prec != 2 && prec != 3) return -1;
  if (bad_trans(TA)) return -2;
  if (bad_trans(TB)) return -3;
  if (M < 0) return -4;
  if (N < 0) return -5;
  if (K < 0) return -6;
  if (lda < std::max(1, TA == kNoTrans ? M : K)) return -9;
  if (ldb < std::max(1, TB == kNoTrans ? K : N)) return -11;
  if (ldc < std::max(1, M)) return -14;
  (prec == 1 ? sgemm_tf32_dev : prec == 2 ? sgemm_bf16_dev : sgemm_tf32x3_dev)(TA == kNoTrans ? kNoTrans : kTrans,
                                                TB == kNoTrans ? kNoTrans : kTrans, M, N, K, alpha,
                                                A, lda, B, ldb, beta, C, ldc, stream(), 0);
  return 0;
}

int atlb_dgemm_batched_dev(int TA, int TB, int count, const int *M, const int *N, const int *K,
                           double alpha, const double *const *A, const int *lda,
                           const double *const *B, const int *ldb, double beta, double *const *C,
                           const int *ldc) {
  if (bad_trans(TA)) return -1;
  if (bad_trans(TB)) return -2;
  if (count < 0) return -3;
  if (count == 0) return 0;
  std::vector<GemmProb> P(count);
  for (int i = 0; i < count; i++) {
    if (M[i] < 0) return -4;
    if (N[i] < 0) return -5;
    if (K[i] < 0) return -6;
    if (lda[i] < std::max(1, TA == kNoTrans ? M[i] : K[i])) return -9;
    if (ldb[i] < std::max(1, TB == kNoTrans ? K[i] : N[i])) return -11;
    if (ldc[i] < std::max(1, M[i])) return -14;
    P[i] = {A[i], B[i], C[i], M[i], N[i], K[i], lda[i], ldb[i], ldc[i], alpha, beta};
  }
  dgemm_grouped_dev(TA == kNoTrans ? kNoTrans : kTrans, TB == kNoTrans ? kNoTrans : kTrans, P.data(),
                    count, stream());
  return 0;
}

int atlb_dtrsm_dev(int Side, int Uplo, int TA, int Diag, int M, int N, double alpha,
                   const double *A, int lda, double *B, int ldb) {
  if (Side != kLeft && Side != kRight) return -1;
  if (Uplo != kUpper && Uplo != kLower) return -2;
  if (bad_trans(TA)) return -3;
  if (Diag != kUnit && Diag != kNonUnit) return -4;
  if (M < 0) return -5;
  if (N < 0) return -6;
  if (lda < std::max(1, Side == kLeft ? M : N)) return -9;
  if (ldb < std::max(1, M)) return -11;
  trsm_dev<double>(Side, Uplo, TA == kNoTrans ? kNoTrans : kTrans, Diag, M, N, alpha, A, lda, B,
                   ldb, stream());
  return 0;
}

int atlb_dsyrk_dev(int Uplo, int Trans, int N, int K, double alpha, const double *A, int lda,
                   double beta, double *C, int ldc) {
  if (Uplo != kUpper && Uplo != kLower) return -1;
  if (bad_trans(Trans)) return -2;
  if (N < 0) return -3;
  if (K < 0) return -4;
  if (lda < std::max(1, Trans == kNoTrans ? N : K)) return -7;
  if (ldc < std::max(1, N)) return -10;
  int tri = Uplo == kLower ? 1 : 2;
  if (Trans == kNoTrans)
    dgemm_dev(kNoTrans, kTrans, N, N, K, alpha, A, lda, A, lda, beta, C, ldc, stream(), tri);
  else
    dgemm_dev(kTrans, kNoTrans, N, N, K, alpha, A, lda, A, lda, beta, C, ldc, stream(), tri);
  return 0;
}

int atlb_dgetrf_dev(int M, int N, double *A, int lda, int *ipiv, int *dinfo) {
  if (M < 0) return -1;
  if (N < 0) return -2;
  if (lda < std::max(1, M)) return -4;
  if (std::min(M, N) == 0) return 0;
  getrf_dev<double>(M, N, A, lda, ipiv, dinfo, stream());
  return 0;
}

int atlb_sgetrf_dev(int M, int N, float *A, int lda, int *ipiv, int *dinfo, int prec) {
  if (M < 0) return -1;
  if (N < 0) return -2;
  if (lda < std::max(1, M)) return -4;
  if (prec < kPrecFP32 || prec > kPrecTF32x3) return -7;
  if (std::min(M, N) == 0) return 0;
  getrf_dev<float>(M, N, A, lda, ipiv, dinfo, stream(), factor_gemm(prec));
  return 0;
}

int atlb_dgetrs_dev(int Trans, int N, int NRHS, const double *A, int lda, const int *ipiv,
                    double *B, int ldb) {
  if (bad_trans(Trans)) return -1;
  if (N < 0) return -2;
  if (NRHS < 0) return -3;
  if (lda < std::max(1, N)) return -5;
  if (ldb < std::max(1, N)) return -8;
  getrs_dev<double>(Trans == kNoTrans ? kNoTrans : kTrans, N, NRHS, A, lda, ipiv, B, ldb,
                    stream());
  return 0;
}

int atlb_dpotrf_dev(int Uplo, int N, double *A, int lda, int *dinfo) {
  if (Uplo != kUpper && Uplo != kLower) return -1;
  if (N < 0) return -2;
  if (lda < std::max(1, N)) return -4;
  if (N == 0) return 0;
  potrf_dev<double>(Uplo, N, A, lda, dinfo, stream());
  return 0;
}

int atlb_dpotrs_dev(int Uplo, int N, int NRHS, const double *A, int lda, double *B, int ldb) {
  if (Uplo != kUpper && Uplo != kLower) return -1;
  if (N < 0) return -2;
  if (NRHS < 0) return -3;
  if (lda < std::max(1, N)) return -5;
  if (ldb < std::max(1, N)) return -7;
  potrs_dev<double>(Uplo, N, NRHS, A, lda, B, ldb, stream());
  return 0;
}

int atlb_dgeqrf_dev(int M, int N, double *A, int lda, double *tau) {
  if (M < 0) return -1;
  if (N < 0) return -2;
  if (lda < std::max(1, M)) return -4;
  if (M == 0 || N == 0) return 0;
  dgeqrf_dev(M, N, A, lda, tau, stream());
  return 0;
}

}  // extern "C"
