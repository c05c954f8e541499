// The rest of the level-3 BLAS and the inverse / least-squares LAPACK routines
// of the reference's C interface, on the GPU kernels of the hot path:
//
//   cblas_dsymm   (interfaces/blas/C/src/cblas_dsymm.c)    symmetric copy + DGEMM
//   cblas_dsyr2k  (interfaces/blas/C/src/cblas_dsyr2k.c)   two triangle-masked DGEMMs
//   cblas_zgemm   (interfaces/blas/C/src/cblas_zgemm.c)    four real DGEMMs on split parts
//   clapack_dgetri (interfaces/lapack/C/src/clapack_dgetri.c, src/lapack/ATL_getri.c)
//   clapack_dtrtri / dlauum / dpotri (clapack_dtrtri.c, clapack_dlauum.c, clapack_dpotri.c,
//                  src/lapack/ATL_trtri.c, ATL_lauum.c)
//   clapack_dgels  (clapack_dgels.c, src/lapack/ATL_gels.c)  QR / LQ least squares
//   clapack_dgelqf (clapack_dgelqf.c)                        LQ = transposed QR
//   ATL_dormqr     (src/lapack/ATL_ormqr.c)                  blocked Q application
//
// Row-major calls are mapped the way the reference maps them: DSYMM swaps side
// and uplo with M and N, DSYR2K flips uplo and trans, ZGEMM swaps operands,
// trtri / lauum / potri flip uplo, getri runs on the column-major view, gels
// flips TA with M and N, gelqf of a row-major matrix is the column-major QR of
// its view.  Entry points take host or device pointers like the rest of the
// C ABI and are synchronous.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "../../include/atlas_b200.h"
#include "staging.h"

namespace atlb {
void xerbla(int pos, const char *rout);

namespace {

void sync_st(cudaStream_t st) { ATLB_CUDA_CHECK(cudaStreamSynchronize(st)); }

int grid_of(long n) { return (int)std::min<long>((n + 255) / 256, 8192); }

// W (n x n, ld n) = I
__global__ void eye_kernel(int n, double *W) {
  const long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x)
    W[idx] = (idx % n) == (idx / n) ? 1.0 : 0.0;
}

// D <- the `uplo` triangle of S (with the diagonal when diag != 0); the rest
// of D is left as it is (zero = 1: set it to zero instead)
__global__ void copy_tri_kernel(int n, int lower, int diag, int zero, const double *S, long lds, double *D,
                                long ldd) {
  const long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const bool in = lower ? (i > j || (diag && i == j)) : (i < j || (diag && i == j));
    if (in) D[i + (long)j * ldd] = S[i + (long)j * lds];
    else if (zero) D[i + (long)j * ldd] = 0.0;
  }
}

// rows r0..r1 of the n-column matrix at B set to zero
__global__ void zero_rows_kernel(int r0, int r1, int n, double *B, long ldb) {
  const int rows = r1 - r0;
  const long total = (long)rows * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x)
    B[r0 + (int)(idx % rows) + (idx / rows) * ldb] = 0.0;
}

// complex (interleaved) rows x cols at Z -> real and imaginary parts (ld rows);
// sign = -1 conjugates
__global__ void zsplit_kernel(int rows, int cols, const double *Z, long ldz, double sign, double *R, double *I) {
  const long total = (long)rows * cols;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % rows), j = (int)(idx / rows);
    const double *z = Z + 2 * (i + (long)j * ldz);
    R[idx] = z[0];
    I[idx] = sign * z[1];
  }
}

// C = alpha * (Pr + i Pi) + beta * C (complex, interleaved); beta == 0: C not read
__global__ void zcombine_kernel(int m, int n, const double *Pr, const double *Pi, double ar, double ai, double br,
                                double bi, double *C, long ldc) {
  const long total = (long)m * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % m), j = (int)(idx / m);
    double *c = C + 2 * (i + (long)j * ldc);
    const double pr = Pr[idx], pi = Pi[idx];
    double cr = ar * pr - ai * pi, ci = ar * pi + ai * pr;
    if (br != 0.0 || bi != 0.0) {
      const double xr = c[0], xi = c[1];
      cr += br * xr - bi * xi;
      ci += br * xi + bi * xr;
    }
    c[0] = cr;
    c[1] = ci;
  }
}

inline int eff_trans(int t) { return t == kNoTrans ? kNoTrans : kTrans; }

// first zero on the diagonal of the n x n matrix at A (1-based), 0 if none
int first_zero_diag(int n, const double *A, long lda, cudaStream_t st) {
  if (n <= 0) return 0;
  double *h = (double *)pinned(kSlotExt3, sizeof(double) * n);
  ATLB_CUDA_CHECK(cudaMemcpy2DAsync(h, sizeof(double), A, (lda + 1) * sizeof(double), sizeof(double), n,
                                    cudaMemcpyDeviceToHost, st));
  sync_st(st);
  for (int i = 0; i < n; i++)
    if (h[i] == 0.0) return i + 1;
  return 0;
}

}  // namespace

// ---------------------------------------------------------------- device routines
void dsymm_dev(int side, int uplo, int M, int N, double alpha, const double *A, long lda, const double *B,
               long ldb, double beta, double *C, long ldc, cudaStream_t st) {
  const int na = side == kLeft ? M : N;
  if (M <= 0 || N <= 0) return;
  double *F = (double *)scratch(kSlotExt0, sizeof(double) * (size_t)na * na);
  symmetrize_dev(uplo, na, A, lda, F, na, st);
  if (side == kLeft) dgemm_dev(kNoTrans, kNoTrans, M, N, M, alpha, F, na, B, ldb, beta, C, ldc, st);
  else dgemm_dev(kNoTrans, kNoTrans, M, N, N, alpha, B, ldb, F, na, beta, C, ldc, st);
}

void dsyr2k_dev(int uplo, int trans, int N, int K, double alpha, const double *A, long lda, const double *B,
                long ldb, double beta, double *C, long ldc, cudaStream_t st) {
  if (N <= 0) return;
  const int tri = uplo == kLower ? 1 : 2;
  if (trans == kNoTrans) {  // alpha A B^T + alpha B A^T
    dgemm_dev(kNoTrans, kTrans, N, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
    dgemm_dev(kNoTrans, kTrans, N, N, K, alpha, B, ldb, A, lda, 1.0, C, ldc, st, tri);
  } else {                  // alpha A^T B + alpha B^T A
    dgemm_dev(kTrans, kNoTrans, N, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
    dgemm_dev(kTrans, kNoTrans, N, N, K, alpha, B, ldb, A, lda, 1.0, C, ldc, st, tri);
  }
}

// C = alpha op(A) op(B) + beta C for complex double (interleaved, leading
// dimensions in complex elements): op(A) = Ar' + i Ai' with Ai' negated for
// ConjTrans, then Re = Ar'Br' - Ai'Bi', Im = Ar'Bi' + Ai'Br' on the DMMA DGEMM.
void zgemm_dev(int ta, int tb, int M, int N, int K, const double *alpha, const double *A, long lda,
               const double *B, long ldb, const double *beta, double *C, long ldc, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  const int ma = ta == kNoTrans ? M : K, ka = ta == kNoTrans ? K : M;
  const int mb = tb == kNoTrans ? K : N, kb = tb == kNoTrans ? N : K;
  const size_t na = (size_t)ma * ka, nb = (size_t)mb * kb, nc = (size_t)M * N;
  double *ws = (double *)scratch(kSlotExt0, sizeof(double) * (2 * na + 2 * nb + 2 * nc + 16));
  double *Ar = ws, *Ai = Ar + na, *Br = Ai + na, *Bi = Br + nb, *Pr = Bi + nb, *Pi = Pr + nc;
  if (K > 0) {
    zsplit_kernel<<<grid_of((long)na), 256, 0, st>>>(ma, ka, A, lda, ta == kConjTrans ? -1.0 : 1.0, Ar, Ai);
    ATLB_CUDA_CHECK(cudaGetLastError());
    zsplit_kernel<<<grid_of((long)nb), 256, 0, st>>>(mb, kb, B, ldb, tb == kConjTrans ? -1.0 : 1.0, Br, Bi);
    ATLB_CUDA_CHECK(cudaGetLastError());
    const int a = eff_trans(ta), b = eff_trans(tb);
    const long la = std::max(ma, 1), lb = std::max(mb, 1);
    dgemm_dev(a, b, M, N, K, 1.0, Ar, la, Br, lb, 0.0, Pr, M, st);
    dgemm_dev(a, b, M, N, K, -1.0, Ai, la, Bi, lb, 1.0, Pr, M, st);
    dgemm_dev(a, b, M, N, K, 1.0, Ar, la, Bi, lb, 0.0, Pi, M, st);
    dgemm_dev(a, b, M, N, K, 1.0, Ai, la, Br, lb, 1.0, Pi, M, st);
  } else {
    ATLB_CUDA_CHECK(cudaMemsetAsync(Pr, 0, sizeof(double) * 2 * nc, st));
  }
  zcombine_kernel<<<grid_of((long)nc), 256, 0, st>>>(M, N, Pr, Pi, alpha[0], alpha[1], beta[0], beta[1], C, ldc);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// A^-1 from getrf's factors: solve A X = I with the factors (getrs), X -> A.
// Returns the first zero pivot of U (1-based; A is then left unchanged).
int dgetri_dev(int N, double *A, long lda, const int *ipiv, cudaStream_t st) {
  if (N <= 0) return 0;
  const int z = first_zero_diag(N, A, lda, st);
  if (z) return z;
  double *W = (double *)scratch(kSlotExt1, sizeof(double) * (size_t)N * N);
  eye_kernel<<<grid_of((long)N * N), 256, 0, st>>>(N, W);
  ATLB_CUDA_CHECK(cudaGetLastError());
  getrs_dev<double>(kNoTrans, N, N, A, lda, ipiv, W, N, st);
  ATLB_CUDA_CHECK(cudaMemcpy2DAsync(A, lda * sizeof(double), W, N * sizeof(double), N * sizeof(double), N,
                                    cudaMemcpyDeviceToDevice, st));
  return 0;
}

// T^-1 in place of the `uplo` triangle of A (the other triangle, and the
// diagonal when unit, are not touched).  Returns the first zero diagonal
// entry (1-based, non-unit only; A then unchanged).
int dtrtri_dev(int uplo, int diag, int N, double *A, long lda, cudaStream_t st) {
  if (N <= 0) return 0;
  if (diag == kNonUnit) {
    const int z = first_zero_diag(N, A, lda, st);
    if (z) return z;
  }
  double *W = (double *)scratch(kSlotExt1, sizeof(double) * (size_t)N * N);
  eye_kernel<<<grid_of((long)N * N), 256, 0, st>>>(N, W);
  ATLB_CUDA_CHECK(cudaGetLastError());
  trsm_dev<double>(kLeft, uplo, kNoTrans, diag, N, N, 1.0, A, lda, W, N, st);
  copy_tri_kernel<<<grid_of((long)N * N), 256, 0, st>>>(N, uplo == kLower, diag == kNonUnit, 0, W, N, A, lda);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

// U U^T (upper) or L^T L (lower) into the same triangle of A
void dlauum_dev(int uplo, int N, double *A, long lda, cudaStream_t st) {
  if (N <= 0) return;
  double *W = (double *)scratch(kSlotExt1, sizeof(double) * (size_t)N * N);
  copy_tri_kernel<<<grid_of((long)N * N), 256, 0, st>>>(N, uplo == kLower, 1, 1, A, lda, W, N);
  ATLB_CUDA_CHECK(cudaGetLastError());
  if (uplo == kUpper) dgemm_dev(kNoTrans, kTrans, N, N, N, 1.0, W, N, W, N, 0.0, A, lda, st, 2);
  else dgemm_dev(kTrans, kNoTrans, N, N, N, 1.0, W, N, W, N, 0.0, A, lda, st, 1);
}

// Least squares / minimum norm with QR or LQ (LAPACK dgels' four cases).  B
// holds max(M, N) rows.  Returns the first zero diagonal of the triangular
// factor (1-based): the system is rank deficient and B is not solved.
int dgels_dev(int trans, int M, int N, int NRHS, double *A, long lda, double *B, long ldb, cudaStream_t st) {
  const int mn = std::min(M, N);
  if (mn == 0) {
    if (NRHS > 0 && std::max(M, N) > 0) {
      zero_rows_kernel<<<grid_of((long)std::max(M, N) * NRHS), 256, 0, st>>>(0, std::max(M, N), NRHS, B, ldb);
      ATLB_CUDA_CHECK(cudaGetLastError());
    }
    return 0;
  }
  double *tau = (double *)scratch(kSlotExt2, sizeof(double) * (size_t)mn);
  const bool tall = M >= N;
  // the matrix whose QR is taken: A itself (M >= N) or A^T (M < N, the LQ case)
  double *Q = A;
  long ldq = lda;
  int qm = M, qn = N;
  if (!tall) {
    Q = (double *)scratch(kSlotExt1, sizeof(double) * (size_t)M * N);
    transpose_dev(M, N, A, lda, Q, N, st);
    ldq = N;
    qm = N;
    qn = M;
  }
  dgeqrf_dev(qm, qn, Q, ldq, tau, st);
  const int z = first_zero_diag(mn, Q, ldq, st);
  int info = 0;
  if (z) {
    info = z;
  } else if (NRHS > 0) {
    const bool ls = (trans == kNoTrans) == tall;  // least squares (else minimum norm)
    if (ls) {  // x = R^-1 (Q^T b)[0:mn]
      dormqr_dev(kLeft, kTrans, qm, NRHS, qn, Q, ldq, tau, B, ldb, st);
      trsm_dev<double>(kLeft, kUpper, kNoTrans, kNonUnit, mn, NRHS, 1.0, Q, ldq, B, ldb, st);
    } else {   // x = Q [R^-T b[0:mn]; 0]
      trsm_dev<double>(kLeft, kUpper, kTrans, kNonUnit, mn, NRHS, 1.0, Q, ldq, B, ldb, st);
      zero_rows_kernel<<<grid_of((long)(qm - mn) * NRHS + 1), 256, 0, st>>>(mn, qm, NRHS, B, ldb);
      ATLB_CUDA_CHECK(cudaGetLastError());
      dormqr_dev(kLeft, kNoTrans, qm, NRHS, qn, Q, ldq, tau, B, ldb, st);
    }
  }
  if (!tall) transpose_dev(N, M, Q, N, A, lda, st);  // A holds its LQ factorization
  return info;
}

}  // namespace atlb

using namespace atlb;

namespace {
bool bad_order(int o) { return o != CblasRowMajor && o != CblasColMajor; }
bool bad_uplo(int u) { return u != CblasUpper && u != CblasLower; }
bool bad_tr(int t) { return t != CblasNoTrans && t != CblasTrans && t != CblasConjTrans; }
int flip_uplo(int u) { return u == CblasUpper ? kLower : kUpper; }
}  // namespace

extern "C" {

void cblas_dsymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side, const enum CBLAS_UPLO Uplo,
                 const int M, const int N, const double alpha, const double *A, const int lda,
                 const double *B, const int ldb, const double beta, double *C, const int ldc) {
  // interfaces/blas/C/src/cblas_dsymm.c: argument positions as there
  int info = 0;
  auto err = [&](int p) { if (!info) info = p; };
  if (bad_order(Order)) err(1);
  if (Side != CblasLeft && Side != CblasRight) err(2);
  if (bad_uplo(Uplo)) err(3);
  if (M < 0) err(4);
  if (N < 0) err(5);
  const int na = Side == CblasLeft ? M : N;
  if (lda < std::max(1, na)) err(8);
  const int rows = Order == CblasColMajor ? M : N;
  if (ldb < std::max(1, rows)) err(10);
  if (ldc < std::max(1, rows)) err(13);
  if (info) { xerbla(info, "cblas_dsymm"); return; }
  if (M == 0 || N == 0) return;
  // row-major: the transposed problem, side and triangle flipped, M and N swapped
  int side = Side, uplo = Uplo, m = M, n = N;
  if (Order == CblasRowMajor) {
    side = Side == CblasLeft ? kRight : kLeft;
    uplo = flip_uplo(Uplo);
    m = N;
    n = M;
  }
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, na, na, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, m, n, ldb, true, st);
  DMat<double> dC = stage_in(kSlotC, (const double *)C, m, n, ldc, beta != 0.0, st);
  dsymm_dev(side, uplo, m, n, alpha, dA.d, dA.ld, dB.d, dB.ld, beta, dC.d, dC.ld, st);
  stage_out(C, ldc, dC, m, n, st);
  sync_st(st);
}

void cblas_dsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE Trans,
                  const int N, const int K, const double alpha, const double *A, const int lda,
                  const double *B, const int ldb, const double beta, double *C, const int ldc) {
  // interfaces/blas/C/src/cblas_dsyr2k.c
  int info = 0;
  auto err = [&](int p) { if (!info) info = p; };
  if (bad_order(Order)) err(1);
  if (bad_uplo(Uplo)) err(2);
  if (bad_tr(Trans)) err(3);
  if (N < 0) err(4);
  if (K < 0) err(5);
  const bool colnt = (Order == CblasColMajor) == (Trans == CblasNoTrans);
  const int ar = colnt ? N : K;  // rows of the stored A and B
  if (lda < std::max(1, ar)) err(8);
  if (ldb < std::max(1, ar)) err(10);
  if (ldc < std::max(1, N)) err(13);
  if (info) { xerbla(info, "cblas_dsyr2k"); return; }
  if (N == 0) return;
  int uplo = Uplo, trans = Trans == CblasNoTrans ? kNoTrans : kTrans;
  if (Order == CblasRowMajor) {
    uplo = flip_uplo(Uplo);
    trans = trans == kNoTrans ? kTrans : kNoTrans;
  }
  const int ac = trans == kNoTrans ? K : N;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, ar, ac, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, ar, ac, ldb, true, st);
  DMat<double> dC = stage_in(kSlotC, (const double *)C, N, N, ldc, true, st);
  dsyr2k_dev(uplo, trans, N, K, alpha, dA.d, dA.ld, dB.d, dB.ld, beta, dC.d, dC.ld, st);
  stage_out(C, ldc, dC, N, N, st);
  sync_st(st);
}

void cblas_zgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta, void *C,
                 const int ldc) {
  // interfaces/blas/C/src/cblas_zgemm.c: positions as cblas_dgemm's
  int info = 0;
  auto err = [&](int p) { if (!info) info = p; };
  if (bad_order(Order)) err(1);
  if (bad_tr(TransA)) err(2);
  if (bad_tr(TransB)) err(3);
  if (M < 0) err(4);
  if (N < 0) err(5);
  if (K < 0) err(6);
  const bool cm = Order == CblasColMajor;
  const int nra = cm ? (TransA == CblasNoTrans ? M : K) : (TransA == CblasNoTrans ? K : M);
  const int nrb = cm ? (TransB == CblasNoTrans ? K : N) : (TransB == CblasNoTrans ? N : K);
  if (lda < std::max(1, nra)) err(9);
  if (ldb < std::max(1, nrb)) err(11);
  if (ldc < std::max(1, cm ? M : N)) err(14);
  // row-major: C^T = op(B)^T op(A)^T, the column-major product with the
  // operands (and their transpose flags) exchanged
  int ta = TransA, tb = TransB, m = M, n = N;
  const void *a = A, *b = B;
  int la = lda, lb = ldb;
  if (!cm) {
    std::swap(ta, tb);
    std::swap(m, n);
    std::swap(a, b);
    std::swap(la, lb);
  }
  const int ma = ta == CblasNoTrans ? m : K, ka = ta == CblasNoTrans ? K : m;
  const int mb = tb == CblasNoTrans ? K : n, kb = tb == CblasNoTrans ? n : K;
  if (info) { xerbla(info, "cblas_zgemm"); return; }
  if (M == 0 || N == 0) return;
  const double *al = (const double *)alpha, *be = (const double *)beta;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, (const double *)a, 2 * ma, ka, 2L * la, true, st);
  DMat<double> dB = stage_in(kSlotB, (const double *)b, 2 * mb, kb, 2L * lb, true, st);
  const bool readc = be[0] != 0.0 || be[1] != 0.0;
  DMat<double> dC = stage_in(kSlotC, (const double *)C, 2 * m, n, 2L * ldc, readc, st);
  zgemm_dev(ta, tb, m, n, K, al, dA.d, dA.ld / 2, dB.d, dB.ld / 2, be, dC.d, dC.ld / 2, st);
  stage_out((double *)C, 2L * ldc, dC, 2 * m, n, st);
  sync_st(st);
}

int clapack_dgetri(const enum CBLAS_ORDER Order, const int N, double *A, const int lda, const int *ipiv) {
  // interfaces/lapack/C/src/clapack_dgetri.c -> src/lapack/ATL_getri.c; the
  // row-major inverse is the column-major one of the view (ATL_getriR)
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (N < 0) ierr = -2;
  else if (lda < std::max(1, N)) ierr = -4;
  if (ierr) { xerbla(-ierr, "clapack_dgetri"); return ierr; }
  if (N == 0) return 0;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  int *dip = stage_vec_in<int>(kSlotIpiv, ipiv, N, true, st);
  const int info = dgetri_dev(N, dA.d, dA.ld, dip, st);
  stage_out(A, lda, dA, N, N, st);
  sync_st(st);
  return info;
}

int clapack_dtrtri(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const enum CBLAS_DIAG Diag,
                   const int N, double *A, const int lda) {
  // interfaces/lapack/C/src/clapack_dtrtri.c.  The reference tests an
  // uninitialised `ierr` before calling ATL_dtrtri; the intended behaviour
  // (invert when the arguments are valid) is implemented.
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (bad_uplo(Uplo)) ierr = -2;
  else if (Diag != CblasUnit && Diag != CblasNonUnit) ierr = -3;
  else if (N < 0) ierr = -4;
  else if (lda < std::max(1, N)) ierr = -6;
  if (ierr) { xerbla(-ierr, "clapack_dtrtri"); return ierr; }
  if (N == 0) return 0;
  const int uplo = Order == CblasRowMajor ? flip_uplo(Uplo) : (int)Uplo;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  const int info = dtrtri_dev(uplo, Diag, N, dA.d, dA.ld, st);
  stage_out(A, lda, dA, N, N, st);
  sync_st(st);
  return info;
}

int clapack_dlauum(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N, double *A,
                   const int lda) {
  // interfaces/lapack/C/src/clapack_dlauum.c
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (bad_uplo(Uplo)) ierr = -2;
  else if (N < 0) ierr = -3;
  else if (lda < std::max(1, N)) ierr = -5;
  if (ierr) { xerbla(-ierr, "clapack_dlauum"); return ierr; }
  if (N == 0) return 0;
  const int uplo = Order == CblasRowMajor ? flip_uplo(Uplo) : (int)Uplo;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  dlauum_dev(uplo, N, dA.d, dA.ld, st);
  stage_out(A, lda, dA, N, N, st);
  sync_st(st);
  return 0;
}

int clapack_dpotri(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N, double *A,
                   const int lda) {
  // interfaces/lapack/C/src/clapack_dpotri.c: trtri (non-unit), then lauum
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (bad_uplo(Uplo)) ierr = -2;
  else if (N < 0) ierr = -3;
  else if (lda < std::max(1, N)) ierr = -5;
  if (ierr) { xerbla(-ierr, "clapack_dpotri"); return ierr; }
  if (N == 0) return 0;
  const int uplo = Order == CblasRowMajor ? flip_uplo(Uplo) : (int)Uplo;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, A, N, N, lda, true, st);
  const int info = dtrtri_dev(uplo, kNonUnit, N, dA.d, dA.ld, st);
  if (!info) dlauum_dev(uplo, N, dA.d, dA.ld, st);
  stage_out(A, lda, dA, N, N, st);
  sync_st(st);
  return info;
}

int clapack_dgels(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA, const int M, const int N,
                  const int NRHS, double *A, const int lda, double *B, const int ldb) {
  // interfaces/lapack/C/src/clapack_dgels.c (its messages name clapack_dgesv;
  // the routine name is reported here)
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (TA != CblasNoTrans && TA != CblasTrans) ierr = -2;
  else if (M < 0) ierr = -3;
  else if (N < 0) ierr = -4;
  else if (NRHS < 0) ierr = -5;
  else if (lda < std::max(1, Order == CblasColMajor ? M : N)) ierr = -7;
  else if (ldb < std::max(1, std::max(M, N))) ierr = -9;
  if (ierr) { xerbla(-ierr, "clapack_dgels"); return ierr; }
  // row-major: the column-major view is A^T (N x M): flip TA, swap M and N
  int ta = TA == CblasNoTrans ? kNoTrans : kTrans, m = M, n = N;
  if (Order == CblasRowMajor) {
    ta = ta == kNoTrans ? kTrans : kNoTrans;
    m = N;
    n = M;
  }
  cudaStream_t st = stream();
  const int rb = std::max(m, n);
  DMat<double> dA = stage_in(kSlotA, A, m, n, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, rb, NRHS, ldb, true, st);
  const int info = dgels_dev(ta, m, n, NRHS, dA.d, dA.ld, dB.d, dB.ld, st);
  stage_out(A, lda, dA, m, n, st);
  stage_out(B, ldb, dB, rb, NRHS, st);
  sync_st(st);
  return info;
}

int clapack_dgelqf(const enum CBLAS_ORDER Order, const int M, const int N, double *A, const int lda,
                   double *TAU) {
  // interfaces/lapack/C/src/clapack_dgelqf.c.  LQ of the column-major M x N
  // matrix = the transposes of the QR factors of A^T (same reflectors and
  // tau); a row-major matrix's LQ is the column-major QR of its N x M view.
  int ierr = 0;
  if (bad_order(Order)) ierr = -1;
  else if (M < 0) ierr = -2;
  else if (N < 0) ierr = -3;
  else if (lda < std::max(1, Order == CblasColMajor ? M : N)) ierr = -5;
  if (ierr) { xerbla(-ierr, "clapack_dgelqf"); return ierr; }
  const int mn = std::min(M, N);
  if (mn == 0) return 0;
  cudaStream_t st = stream();
  double *dtau = stage_vec_in<double>(kSlotTau, TAU, mn, false, st);
  if (Order == CblasRowMajor) {
    DMat<double> dV = stage_in(kSlotA, A, N, M, lda, true, st);
    dgeqrf_dev(N, M, dV.d, dV.ld, dtau, st);
    stage_out(A, lda, dV, N, M, st);
  } else {
    DMat<double> dA = stage_in(kSlotA, A, M, N, lda, true, st);
    double *T = (double *)scratch(kSlotExt1, sizeof(double) * (size_t)M * N);
    transpose_dev(M, N, dA.d, dA.ld, T, N, st);
    dgeqrf_dev(N, M, T, N, dtau, st);
    transpose_dev(N, M, T, N, dA.d, dA.ld, st);
    stage_out(A, lda, dA, M, N, st);
  }
  stage_vec_out<double>(TAU, dtau, mn, st);
  sync_st(st);
  return 0;
}

int ATL_dormqr(const enum CBLAS_SIDE SIDE, const enum CBLAS_TRANSPOSE TRANS, const int M, const int N,
               const int K, double *A, const int lda, const double *TAU, double *C, const int ldc, double *WORK,
               const int LWORK) {
  // src/lapack/ATL_ormqr.c:24-34 (LWORK < 0: workspace query, size in WORK[0];
  // the GPU path keeps its own workspace)
  const int nq = SIDE == CblasLeft ? M : N;
  if (LWORK < 0) {
    if (WORK) *WORK = (double)std::max(1, (SIDE == CblasLeft ? N : M) * 32);
    return 0;
  }
  int ierr = 0;
  if (SIDE != CblasLeft && SIDE != CblasRight) ierr = -1;
  else if (TRANS != CblasNoTrans && TRANS != CblasTrans) ierr = -2;
  else if (M < 0) ierr = -3;
  else if (N < 0) ierr = -4;
  else if (K < 0 || K > nq) ierr = -5;
  else if (lda < std::max(1, nq)) ierr = -7;
  else if (ldc < std::max(1, M)) ierr = -10;
  if (ierr) { xerbla(-ierr, "ATL_dormqr"); return ierr; }
  if (M == 0 || N == 0 || K == 0) return 0;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, (const double *)A, nq, K, lda, true, st);
  double *dtau = stage_vec_in<double>(kSlotTau, TAU, K, true, st);
  DMat<double> dC = stage_in(kSlotC, (const double *)C, M, N, ldc, true, st);
  dormqr_dev(SIDE, TRANS == CblasNoTrans ? kNoTrans : kTrans, M, N, K, dA.d, dA.ld, dtau, dC.d, dC.ld, st);
  stage_out(C, ldc, dC, M, N, st);
  sync_st(st);
  return 0;
}

int atlb_dormqr_dev(int Side, int Trans, int M, int N, int K, const double *A, int lda, const double *tau,
                    double *C, int ldc) {
  const int nq = Side == kLeft ? M : N;
  if (Side != kLeft && Side != kRight) return -1;
  if (Trans != kNoTrans && Trans != kTrans) return -2;
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0 || K > nq) return -5;
  if (lda < std::max(1, nq)) return -7;
  if (ldc < std::max(1, M)) return -10;
  dormqr_dev(Side, Trans, M, N, K, A, lda, tau, C, ldc, stream());
  return 0;
}

}  // extern "C"
