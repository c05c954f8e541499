/* Test infrastructure only (the CPU oracle's pinning recipe, never linked by
 * the library).  The reference's LAPACK sources call the level-1/2/3 BLAS
 * through the CBLAS names and a few ATL_d* internals.  A full ATLAS build
 * routes those to its tuned kernels, which need the install-time search; here
 * they are routed to the reference's own C reference BLAS
 * (src/blas/reference/level{1,2,3}/ATL_dref*.c, compiled unmodified next to
 * this file).  Row-major GEMM and TRSM calls (issued by the row-major LU,
 * ATL_getrfR) are mapped to the column-major reference routines the way CBLAS
 * defines them (operands of the transposed problem); every other routine
 * takes column-major calls only and aborts otherwise, so a call this shim
 * does not cover cannot go unnoticed. */
#include <stdio.h>
#include <stdlib.h>
#include "atlas_enum.h"
#include "atlas_reflevel1.h"
#include "atlas_reflevel2.h"
#include "atlas_reflevel3.h"

static void colmajor(int order, const char *rout)
{
   if (order != CblasColMajor)
   {
      fprintf(stderr, "refcblas: %s called with order %d (only column-major)\n", rout, order);
      abort();
   }
}

void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_TRANSPOSE TB, const int M, const int N, const int K,
                 const double alpha, const double *A, const int lda, const double *B,
                 const int ldb, const double beta, double *C, const int ldc)
{
   if (M <= 0 || N <= 0) return;
   if (Order == CblasRowMajor)
   {  /* C^T = op(B)^T op(A)^T in column-major terms */
      ATL_drefgemm((enum ATLAS_TRANS)TB, (enum ATLAS_TRANS)TA, N, M, K, alpha, B, ldb, A, lda,
                   beta, C, ldc);
      return;
   }
   colmajor(Order, "cblas_dgemm");
   ATL_drefgemm((enum ATLAS_TRANS)TA, (enum ATLAS_TRANS)TB, M, N, K, alpha, A, lda, B, ldb,
                beta, C, ldc);
}

void cblas_dtrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb)
{
   if (M <= 0 || N <= 0) return;
   if (Order == CblasRowMajor)
   {  /* the transposed problem: side and triangle flip, M and N swap */
      ATL_dreftrsm(Side == CblasLeft ? AtlasRight : AtlasLeft,
                   Uplo == CblasUpper ? AtlasLower : AtlasUpper, (enum ATLAS_TRANS)TA,
                   (enum ATLAS_DIAG)Diag, N, M, alpha, A, lda, B, ldb);
      return;
   }
   colmajor(Order, "cblas_dtrsm");
   ATL_dreftrsm((enum ATLAS_SIDE)Side, (enum ATLAS_UPLO)Uplo, (enum ATLAS_TRANS)TA,
                (enum ATLAS_DIAG)Diag, M, N, alpha, A, lda, B, ldb);
}

void cblas_dtrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb)
{
   colmajor(Order, "cblas_dtrmm");
   if (M <= 0 || N <= 0) return;
   ATL_dreftrmm((enum ATLAS_SIDE)Side, (enum ATLAS_UPLO)Uplo, (enum ATLAS_TRANS)TA,
                (enum ATLAS_DIAG)Diag, M, N, alpha, A, lda, B, ldb);
}

void cblas_dsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const double *A, const int lda, const double beta, double *C, const int ldc)
{
   colmajor(Order, "cblas_dsyrk");
   if (N <= 0) return;
   ATL_drefsyrk((enum ATLAS_UPLO)Uplo, (enum ATLAS_TRANS)Trans, N, K, alpha, A, lda, beta, C, ldc);
}

void cblas_dgemv(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA, const int M,
                 const int N, const double alpha, const double *A, const int lda,
                 const double *X, const int incX, const double beta, double *Y, const int incY)
{
   colmajor(Order, "cblas_dgemv");
   if (M <= 0 || N <= 0) return;
   /* ATL_drefgemv takes the dimensions of op(A), CBLAS those of A */
   if (TA == CblasNoTrans)
      ATL_drefgemv(AtlasNoTrans, M, N, alpha, A, lda, X, incX, beta, Y, incY);
   else
      ATL_drefgemv(AtlasTrans, N, M, alpha, A, lda, X, incX, beta, Y, incY);
}

void cblas_dtrsv(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE TA, const enum CBLAS_DIAG Diag, const int N,
                 const double *A, const int lda, double *X, const int incX)
{
   colmajor(Order, "cblas_dtrsv");
   if (N <= 0) return;
   ATL_dreftrsv((enum ATLAS_UPLO)Uplo, (enum ATLAS_TRANS)TA, (enum ATLAS_DIAG)Diag, N, A, lda,
                X, incX);
}

void cblas_dger(const enum CBLAS_ORDER Order, const int M, const int N, const double alpha,
                const double *X, const int incX, const double *Y, const int incY, double *A,
                const int lda)
{
   colmajor(Order, "cblas_dger");
   if (M <= 0 || N <= 0) return;
   ATL_drefger(M, N, alpha, X, incX, Y, incY, A, lda);
}

void ATL_dger(const int M, const int N, const double alpha, const double *X, const int incX,
              const double *Y, const int incY, double *A, const int lda)
{
   if (M <= 0 || N <= 0) return;
   ATL_drefger(M, N, alpha, X, incX, Y, incY, A, lda);
}

int cblas_idamax(const int N, const double *X, const int incX)
{
   if (N <= 0 || incX <= 0) return 0;
   return ATL_idrefamax(N, X, incX);
}

void cblas_dscal(const int N, const double alpha, double *X, const int incX)
{
   if (N <= 0 || incX <= 0) return;
   ATL_drefscal(N, alpha, X, incX);
}

void cblas_dswap(const int N, double *X, const int incX, double *Y, const int incY)
{
   if (N <= 0) return;
   ATL_drefswap(N, X, incX, Y, incY);
}

void cblas_dcopy(const int N, const double *X, const int incX, double *Y, const int incY)
{
   if (N <= 0) return;
   ATL_drefcopy(N, X, incX, Y, incY);
}

double cblas_ddot(const int N, const double *X, const int incX, const double *Y, const int incY)
{
   if (N <= 0) return 0.0;
   return ATL_drefdot(N, X, incX, Y, incY);
}

double cblas_dnrm2(const int N, const double *X, const int incX)
{
   if (N <= 0 || incX <= 0) return 0.0;
   return ATL_drefnrm2(N, X, incX);
}
