// Fortran 77 calling convention for the same routines (the reference's
// interfaces/blas/F77/src/*.f and interfaces/lapack/F77/src/*.f): every
// argument by address, characters as the first letter (upper or lower case;
// trailing hidden string lengths are not read), column-major arrays, 1-based
// pivot indices, INFO returned through its argument.  Argument errors are
// reported with the F77 routine's argument positions through the library's
// xerbla (message, then exit unless the error mode is "return", in which case
// INFO = -position for the LAPACK routines).  Each routine forwards to the C
// entry point of the same operation after its checks; IPIV must be host
// memory (it is converted between 0- and 1-based numbering on the host).
#include <algorithm>
#include <cctype>
#include <vector>
#include "common.cuh"
#include "../../include/atlas_b200.h"

namespace atlb {
void xerbla(int pos, const char *rout);
}
using atlb::xerbla;

namespace {
int up(const char *c) { return std::toupper((unsigned char)c[0]); }
int f_trans(const char *c) {  // 0 when invalid
  switch (up(c)) {
    case 'N': return CblasNoTrans;
    case 'T': return CblasTrans;
    case 'C': return CblasConjTrans;
  }
  return 0;
}
int f_uplo(const char *c) { return up(c) == 'U' ? CblasUpper : up(c) == 'L' ? CblasLower : 0; }
int f_side(const char *c) { return up(c) == 'L' ? CblasLeft : up(c) == 'R' ? CblasRight : 0; }
int f_diag(const char *c) { return up(c) == 'U' ? CblasUnit : up(c) == 'N' ? CblasNonUnit : 0; }
int mx1(int a) { return std::max(1, a); }

// LAPACK-style report: INFO = -pos, xerbla(pos)
void lapack_err(int pos, const char *rout, int *info) {
  *info = -pos;
  xerbla(pos, rout);
}
}  // namespace

extern "C" {

// interfaces/blas/F77/src/dgemm.f
void dgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const double *alpha,
            const double *a, const int *lda, const double *b, const int *ldb, const double *beta, double *c,
            const int *ldc) {
  const int ta = f_trans(transa), tb = f_trans(transb);
  int info = 0;
  if (!ta) info = 1;
  else if (!tb) info = 2;
  else if (*m < 0) info = 3;
  else if (*n < 0) info = 4;
  else if (*k < 0) info = 5;
  else if (*lda < mx1(ta == CblasNoTrans ? *m : *k)) info = 8;
  else if (*ldb < mx1(tb == CblasNoTrans ? *k : *n)) info = 10;
  else if (*ldc < mx1(*m)) info = 13;
  if (info) { xerbla(info, "DGEMM "); return; }
  cblas_dgemm(CblasColMajor, (CBLAS_TRANSPOSE)ta, (CBLAS_TRANSPOSE)tb, *m, *n, *k, *alpha, a, *lda, b, *ldb,
              *beta, c, *ldc);
}

// interfaces/blas/F77/src/sgemm.f
void sgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const float *alpha,
            const float *a, const int *lda, const float *b, const int *ldb, const float *beta, float *c,
            const int *ldc) {
  const int ta = f_trans(transa), tb = f_trans(transb);
  int info = 0;
  if (!ta) info = 1;
  else if (!tb) info = 2;
  else if (*m < 0) info = 3;
  else if (*n < 0) info = 4;
  else if (*k < 0) info = 5;
  else if (*lda < mx1(ta == CblasNoTrans ? *m : *k)) info = 8;
  else if (*ldb < mx1(tb == CblasNoTrans ? *k : *n)) info = 10;
  else if (*ldc < mx1(*m)) info = 13;
  if (info) { xerbla(info, "SGEMM "); return; }
  cblas_sgemm(CblasColMajor, (CBLAS_TRANSPOSE)ta, (CBLAS_TRANSPOSE)tb, *m, *n, *k, *alpha, a, *lda, b, *ldb,
              *beta, c, *ldc);
}

// interfaces/blas/F77/src/zgemm.f (complex*16 alpha, beta: two doubles each)
void zgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const double *alpha,
            const double *a, const int *lda, const double *b, const int *ldb, const double *beta, double *c,
            const int *ldc) {
  const int ta = f_trans(transa), tb = f_trans(transb);
  int info = 0;
  if (!ta) info = 1;
  else if (!tb) info = 2;
  else if (*m < 0) info = 3;
  else if (*n < 0) info = 4;
  else if (*k < 0) info = 5;
  else if (*lda < mx1(ta == CblasNoTrans ? *m : *k)) info = 8;
  else if (*ldb < mx1(tb == CblasNoTrans ? *k : *n)) info = 10;
  else if (*ldc < mx1(*m)) info = 13;
  if (info) { xerbla(info, "ZGEMM "); return; }
  cblas_zgemm(CblasColMajor, (CBLAS_TRANSPOSE)ta, (CBLAS_TRANSPOSE)tb, *m, *n, *k, alpha, a, *lda, b, *ldb, beta,
              c, *ldc);
}

// interfaces/blas/F77/src/dtrsm.f
void dtrsm_(const char *side, const char *uplo, const char *transa, const char *diag, const int *m, const int *n,
            const double *alpha, const double *a, const int *lda, double *b, const int *ldb) {
  const int sd = f_side(side), ul = f_uplo(uplo), ta = f_trans(transa), dg = f_diag(diag);
  int info = 0;
  if (!sd) info = 1;
  else if (!ul) info = 2;
  else if (!ta) info = 3;
  else if (!dg) info = 4;
  else if (*m < 0) info = 5;
  else if (*n < 0) info = 6;
  else if (*lda < mx1(sd == CblasLeft ? *m : *n)) info = 9;
  else if (*ldb < mx1(*m)) info = 11;
  if (info) { xerbla(info, "DTRSM "); return; }
  cblas_dtrsm(CblasColMajor, (CBLAS_SIDE)sd, (CBLAS_UPLO)ul, (CBLAS_TRANSPOSE)ta, (CBLAS_DIAG)dg, *m, *n, *alpha,
              a, *lda, b, *ldb);
}

// interfaces/blas/F77/src/dtrmm.f
void dtrmm_(const char *side, const char *uplo, const char *transa, const char *diag, const int *m, const int *n,
            const double *alpha, const double *a, const int *lda, double *b, const int *ldb) {
  const int sd = f_side(side), ul = f_uplo(uplo), ta = f_trans(transa), dg = f_diag(diag);
  int info = 0;
  if (!sd) info = 1;
  else if (!ul) info = 2;
  else if (!ta) info = 3;
  else if (!dg) info = 4;
  else if (*m < 0) info = 5;
  else if (*n < 0) info = 6;
  else if (*lda < mx1(sd == CblasLeft ? *m : *n)) info = 9;
  else if (*ldb < mx1(*m)) info = 11;
  if (info) { xerbla(info, "DTRMM "); return; }
  cblas_dtrmm(CblasColMajor, (CBLAS_SIDE)sd, (CBLAS_UPLO)ul, (CBLAS_TRANSPOSE)ta, (CBLAS_DIAG)dg, *m, *n, *alpha,
              a, *lda, b, *ldb);
}

// interfaces/blas/F77/src/dsyrk.f
void dsyrk_(const char *uplo, const char *trans, const int *n, const int *k, const double *alpha, const double *a,
            const int *lda, const double *beta, double *c, const int *ldc) {
  const int ul = f_uplo(uplo), tr = f_trans(trans);
  int info = 0;
  if (!ul) info = 1;
  else if (!tr) info = 2;
  else if (*n < 0) info = 3;
  else if (*k < 0) info = 4;
  else if (*lda < mx1(tr == CblasNoTrans ? *n : *k)) info = 7;
  else if (*ldc < mx1(*n)) info = 10;
  if (info) { xerbla(info, "DSYRK "); return; }
  cblas_dsyrk(CblasColMajor, (CBLAS_UPLO)ul, (CBLAS_TRANSPOSE)tr, *n, *k, *alpha, a, *lda, *beta, c, *ldc);
}

// interfaces/blas/F77/src/dsymm.f
void dsymm_(const char *side, const char *uplo, const int *m, const int *n, const double *alpha, const double *a,
            const int *lda, const double *b, const int *ldb, const double *beta, double *c, const int *ldc) {
  const int sd = f_side(side), ul = f_uplo(uplo);
  int info = 0;
  if (!sd) info = 1;
  else if (!ul) info = 2;
  else if (*m < 0) info = 3;
  else if (*n < 0) info = 4;
  else if (*lda < mx1(sd == CblasLeft ? *m : *n)) info = 7;
  else if (*ldb < mx1(*m)) info = 9;
  else if (*ldc < mx1(*m)) info = 12;
  if (info) { xerbla(info, "DSYMM "); return; }
  cblas_dsymm(CblasColMajor, (CBLAS_SIDE)sd, (CBLAS_UPLO)ul, *m, *n, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

// interfaces/blas/F77/src/dsyr2k.f
void dsyr2k_(const char *uplo, const char *trans, const int *n, const int *k, const double *alpha, const double *a,
             const int *lda, const double *b, const int *ldb, const double *beta, double *c, const int *ldc) {
  const int ul = f_uplo(uplo), tr = f_trans(trans);
  int info = 0;
  if (!ul) info = 1;
  else if (!tr) info = 2;
  else if (*n < 0) info = 3;
  else if (*k < 0) info = 4;
  else if (*lda < mx1(tr == CblasNoTrans ? *n : *k)) info = 7;
  else if (*ldb < mx1(tr == CblasNoTrans ? *n : *k)) info = 9;
  else if (*ldc < mx1(*n)) info = 12;
  if (info) { xerbla(info, "DSYR2K"); return; }
  cblas_dsyr2k(CblasColMajor, (CBLAS_UPLO)ul, (CBLAS_TRANSPOSE)tr, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c,
               *ldc);
}

// interfaces/lapack/F77/src/dgetrf.f
void dgetrf_(const int *m, const int *n, double *a, const int *lda, int *ipiv, int *info) {
  *info = 0;
  if (*m < 0) return lapack_err(1, "DGETRF", info);
  if (*n < 0) return lapack_err(2, "DGETRF", info);
  if (*lda < mx1(*m)) return lapack_err(4, "DGETRF", info);
  *info = clapack_dgetrf(CblasColMajor, *m, *n, a, *lda, ipiv);
  for (int i = 0, mn = std::min(*m, *n); i < mn; i++) ipiv[i] += 1;
}

// interfaces/lapack/F77/src/dgetrs.f
void dgetrs_(const char *trans, const int *n, const int *nrhs, const double *a, const int *lda, const int *ipiv,
             double *b, const int *ldb, int *info) {
  const int tr = f_trans(trans);
  *info = 0;
  if (!tr) return lapack_err(1, "DGETRS", info);
  if (*n < 0) return lapack_err(2, "DGETRS", info);
  if (*nrhs < 0) return lapack_err(3, "DGETRS", info);
  if (*lda < mx1(*n)) return lapack_err(5, "DGETRS", info);
  if (*ldb < mx1(*n)) return lapack_err(8, "DGETRS", info);
  std::vector<int> p0(std::max(*n, 1));
  for (int i = 0; i < *n; i++) p0[i] = ipiv[i] - 1;
  *info = clapack_dgetrs(CblasColMajor, (CBLAS_TRANSPOSE)tr, *n, *nrhs, a, *lda, p0.data(), b, *ldb);
}

// interfaces/lapack/F77/src/dgesv.f
void dgesv_(const int *n, const int *nrhs, double *a, const int *lda, int *ipiv, double *b, const int *ldb,
            int *info) {
  *info = 0;
  if (*n < 0) return lapack_err(1, "DGESV ", info);
  if (*nrhs < 0) return lapack_err(2, "DGESV ", info);
  if (*lda < mx1(*n)) return lapack_err(4, "DGESV ", info);
  if (*ldb < mx1(*n)) return lapack_err(7, "DGESV ", info);
  *info = clapack_dgesv(CblasColMajor, *n, *nrhs, a, *lda, ipiv, b, *ldb);
  for (int i = 0; i < *n; i++) ipiv[i] += 1;
}

// interfaces/lapack/F77/src/dgetri.f (LWORK = -1: workspace query)
void dgetri_(const int *n, double *a, const int *lda, const int *ipiv, double *work, const int *lwork, int *info) {
  *info = 0;
  if (*n < 0) return lapack_err(1, "DGETRI", info);
  if (*lda < mx1(*n)) return lapack_err(3, "DGETRI", info);
  if (*lwork == -1) {
    work[0] = mx1(*n);
    return;
  }
  if (*lwork < mx1(*n)) return lapack_err(6, "DGETRI", info);
  std::vector<int> p0(std::max(*n, 1));
  for (int i = 0; i < *n; i++) p0[i] = ipiv[i] - 1;
  *info = clapack_dgetri(CblasColMajor, *n, a, *lda, p0.data());
}

// interfaces/lapack/F77/src/dpotrf.f
void dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
  const int ul = f_uplo(uplo);
  *info = 0;
  if (!ul) return lapack_err(1, "DPOTRF", info);
  if (*n < 0) return lapack_err(2, "DPOTRF", info);
  if (*lda < mx1(*n)) return lapack_err(4, "DPOTRF", info);
  *info = clapack_dpotrf(CblasColMajor, (CBLAS_UPLO)ul, *n, a, *lda);
}

// interfaces/lapack/F77/src/dpotrs.f
void dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda, double *b,
             const int *ldb, int *info) {
  const int ul = f_uplo(uplo);
  *info = 0;
  if (!ul) return lapack_err(1, "DPOTRS", info);
  if (*n < 0) return lapack_err(2, "DPOTRS", info);
  if (*nrhs < 0) return lapack_err(3, "DPOTRS", info);
  if (*lda < mx1(*n)) return lapack_err(5, "DPOTRS", info);
  if (*ldb < mx1(*n)) return lapack_err(7, "DPOTRS", info);
  *info = clapack_dpotrs(CblasColMajor, (CBLAS_UPLO)ul, *n, *nrhs, a, *lda, b, *ldb);
}

// interfaces/lapack/F77/src/dposv.f
void dposv_(const char *uplo, const int *n, const int *nrhs, double *a, const int *lda, double *b, const int *ldb,
            int *info) {
  const int ul = f_uplo(uplo);
  *info = 0;
  if (!ul) return lapack_err(1, "DPOSV ", info);
  if (*n < 0) return lapack_err(2, "DPOSV ", info);
  if (*nrhs < 0) return lapack_err(3, "DPOSV ", info);
  if (*lda < mx1(*n)) return lapack_err(5, "DPOSV ", info);
  if (*ldb < mx1(*n)) return lapack_err(7, "DPOSV ", info);
  *info = clapack_dposv(CblasColMajor, (CBLAS_UPLO)ul, *n, *nrhs, a, *lda, b, *ldb);
}

// interfaces/lapack/F77/src/dpotri.f
void dpotri_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
  const int ul = f_uplo(uplo);
  *info = 0;
  if (!ul) return lapack_err(1, "DPOTRI", info);
  if (*n < 0) return lapack_err(2, "DPOTRI", info);
  if (*lda < mx1(*n)) return lapack_err(4, "DPOTRI", info);
  *info = clapack_dpotri(CblasColMajor, (CBLAS_UPLO)ul, *n, a, *lda);
}

// interfaces/lapack/F77/src/dtrtri.f
void dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info) {
  const int ul = f_uplo(uplo), dg = f_diag(diag);
  *info = 0;
  if (!ul) return lapack_err(1, "DTRTRI", info);
  if (!dg) return lapack_err(2, "DTRTRI", info);
  if (*n < 0) return lapack_err(3, "DTRTRI", info);
  if (*lda < mx1(*n)) return lapack_err(5, "DTRTRI", info);
  *info = clapack_dtrtri(CblasColMajor, (CBLAS_UPLO)ul, (CBLAS_DIAG)dg, *n, a, *lda);
}

// interfaces/lapack/F77/src/dlauum.f
void dlauum_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
  const int ul = f_uplo(uplo);
  *info = 0;
  if (!ul) return lapack_err(1, "DLAUUM", info);
  if (*n < 0) return lapack_err(2, "DLAUUM", info);
  if (*lda < mx1(*n)) return lapack_err(4, "DLAUUM", info);
  *info = clapack_dlauum(CblasColMajor, (CBLAS_UPLO)ul, *n, a, *lda);
}

// interfaces/lapack/F77/src/dgeqrf.f (LWORK = -1: workspace query)
void dgeqrf_(const int *m, const int *n, double *a, const int *lda, double *tau, double *work, const int *lwork,
             int *info) {
  *info = 0;
  if (*m < 0) return lapack_err(1, "DGEQRF", info);
  if (*n < 0) return lapack_err(2, "DGEQRF", info);
  if (*lda < mx1(*m)) return lapack_err(4, "DGEQRF", info);
  if (*lwork == -1) {
    work[0] = mx1(*n) * 32;
    return;
  }
  if (*lwork < mx1(*n)) return lapack_err(7, "DGEQRF", info);
  *info = clapack_dgeqrf(CblasColMajor, *m, *n, a, *lda, tau);
}

// interfaces/lapack/F77/src/dgelqf.f (LWORK = -1: workspace query)
void dgelqf_(const int *m, const int *n, double *a, const int *lda, double *tau, double *work, const int *lwork,
             int *info) {
  *info = 0;
  if (*m < 0) return lapack_err(1, "DGELQF", info);
  if (*n < 0) return lapack_err(2, "DGELQF", info);
  if (*lda < mx1(*m)) return lapack_err(4, "DGELQF", info);
  if (*lwork == -1) {
    work[0] = mx1(*m) * 32;
    return;
  }
  if (*lwork < mx1(*m)) return lapack_err(7, "DGELQF", info);
  *info = clapack_dgelqf(CblasColMajor, *m, *n, a, *lda, tau);
}

// interfaces/lapack/F77/src/dgels.f (LWORK = -1: workspace query)
void dgels_(const char *trans, const int *m, const int *n, const int *nrhs, double *a, const int *lda, double *b,
            const int *ldb, double *work, const int *lwork, int *info) {
  const int tr = f_trans(trans);
  *info = 0;
  if (tr != CblasNoTrans && tr != CblasTrans) return lapack_err(1, "DGELS ", info);
  if (*m < 0) return lapack_err(2, "DGELS ", info);
  if (*n < 0) return lapack_err(3, "DGELS ", info);
  if (*nrhs < 0) return lapack_err(4, "DGELS ", info);
  if (*lda < mx1(*m)) return lapack_err(6, "DGELS ", info);
  if (*ldb < mx1(std::max(*m, *n))) return lapack_err(8, "DGELS ", info);
  const int mn = std::min(*m, *n), need = std::max(1, mn + std::max(mn, *nrhs));
  if (*lwork == -1) {
    work[0] = need * 32;
    return;
  }
  if (*lwork < need) return lapack_err(10, "DGELS ", info);
  *info = clapack_dgels(CblasColMajor, (CBLAS_TRANSPOSE)tr, *m, *n, *nrhs, a, *lda, b, *ldb);
}

}  // extern "C"
