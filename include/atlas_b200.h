/*
 * atlas_b200.h -- C ABI of libatlas_b200.so, a B200 (sm_100a) implementation
 * of ATLAS's dense level-3 BLAS / LAPACK hot path.
 *
 * Part 1 declares the drop-in entry points with the reference's exact
 * prototypes (each comment names the reference declaration it replaces).
 * They take host pointers (device pointers are also accepted and used in
 * place), compute on the GPU and return when the result is in the caller's
 * buffers, like the CPU library.  Argument errors follow cblas_xerbla: a
 * message on stderr and exit(-1), unless atlb_set_error_mode(1) (or the
 * environment variable ATLAS_B200_XERBLA=return) makes them return instead.
 *
 * Part 2 declares extensions with no counterpart in the reference:
 * device-pointer variants (asynchronous on the library's stream), the
 * mixed-precision solvers, the split-integer (Ozaki) DGEMM, batched
 * factorizations and the adjoints of potrf/potrs and getrf/getrs.
 */
#ifndef ATLAS_B200_H
#define ATLAS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef CBLAS_ENUM_DEFINED_H
#define CBLAS_ENUM_DEFINED_H
/* include/cblas.h:5-10 of the reference */
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113, AtlasConj = 114 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
#endif

/* ---------------------------------------------------------------- Part 1 */

/* cblas_dgemm: include/cblas.h:471, interfaces/blas/C/src/cblas_dgemm.c:16-134 */
void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const double alpha, const double *A, const int lda, const double *B,
                 const int ldb, const double beta, double *C, const int ldc);
/* cblas_sgemm: include/cblas.h:441, interfaces/blas/C/src/cblas_sgemm.c:131-133 */
void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc);
/* cblas_dtrsm: include/cblas.h:495, interfaces/blas/C/src/cblas_dtrsm.c:14-105 */
void cblas_dtrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb);
/* cblas_dtrmm: include/cblas.h:490, interfaces/blas/C/src/cblas_dtrmm.c:14 (used by larfb) */
void cblas_dtrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb);
/* cblas_dsyrk: include/cblas.h:481, interfaces/blas/C/src/cblas_dsyrk.c:14-90 */
void cblas_dsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const double *A, const int lda, const double beta, double *C, const int ldc);

/* clapack_dgetrf: include/clapack.h:63, interfaces/lapack/C/src/clapack_dgetrf.c:13-88 */
int clapack_dgetrf(const enum CBLAS_ORDER Order, const int M, const int N, double *A,
                   const int lda, int *ipiv);
/* clapack_dgetrs: include/clapack.h:65, interfaces/lapack/C/src/clapack_dgetrs.c:57 */
int clapack_dgetrs(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE Trans, const int N,
                   const int NRHS, const double *A, const int lda, const int *ipiv, double *B,
                   const int ldb);
/* clapack_dgesv: include/clapack.h:60, interfaces/lapack/C/src/clapack_dgesv.c:61-62 */
int clapack_dgesv(const enum CBLAS_ORDER Order, const int N, const int NRHS, double *A,
                  const int lda, int *ipiv, double *B, const int ldb);
/* clapack_dpotrf: include/clapack.h:74, interfaces/lapack/C/src/clapack_dpotrf.c:43 */
int clapack_dpotrf(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                   double *A, const int lda);
/* clapack_dpotrs: include/clapack.h:76, interfaces/lapack/C/src/clapack_dpotrs.c:56 */
int clapack_dpotrs(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                   const int NRHS, const double *A, const int lda, double *B, const int ldb);
/* clapack_dposv: include/clapack.h:71, interfaces/lapack/C/src/clapack_dposv.c:57-58 */
int clapack_dposv(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N,
                  const int NRHS, double *A, const int lda, double *B, const int ldb);
/* clapack_dgeqrf: include/clapack.h:96, interfaces/lapack/C/src/clapack_dgeqrf.c:14-61 */
int clapack_dgeqrf(const enum CBLAS_ORDER Order, const int M, const int N, double *A,
                   const int lda, double *TAU);
/* ATL_dgeqrf: src/lapack/ATL_geqrf.c:29-196 (LWORK < 0: workspace query) */
int ATL_dgeqrf(const int M, const int N, double *A, const int lda, double *TAU, double *WORK,
               const int LWORK);

/* cblas_dsymm: include/cblas.h, interfaces/blas/C/src/cblas_dsymm.c */
void cblas_dsymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side, const enum CBLAS_UPLO Uplo,
                 const int M, const int N, const double alpha, const double *A, const int lda,
                 const double *B, const int ldb, const double beta, double *C, const int ldc);
/* cblas_dsyr2k: include/cblas.h, interfaces/blas/C/src/cblas_dsyr2k.c */
void cblas_dsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE Trans,
                  const int N, const int K, const double alpha, const double *A, const int lda,
                  const double *B, const int ldb, const double beta, double *C, const int ldc);
/* cblas_zgemm: include/cblas.h, interfaces/blas/C/src/cblas_zgemm.c (complex
 * double, interleaved; alpha and beta point to two doubles) */
void cblas_zgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta, void *C,
                 const int ldc);
/* clapack_dgetri: include/clapack.h:69, interfaces/lapack/C/src/clapack_dgetri.c */
int clapack_dgetri(const enum CBLAS_ORDER Order, const int N, double *A, const int lda, const int *ipiv);
/* clapack_dpotri: include/clapack.h:79, interfaces/lapack/C/src/clapack_dpotri.c */
int clapack_dpotri(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N, double *A,
                   const int lda);
/* clapack_dlauum: include/clapack.h:81, interfaces/lapack/C/src/clapack_dlauum.c */
int clapack_dlauum(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const int N, double *A,
                   const int lda);
/* clapack_dtrtri: include/clapack.h:83, interfaces/lapack/C/src/clapack_dtrtri.c */
int clapack_dtrtri(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo, const enum CBLAS_DIAG Diag,
                   const int N, double *A, const int lda);
/* clapack_dgels: include/clapack.h:86, interfaces/lapack/C/src/clapack_dgels.c */
int clapack_dgels(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TA, const int M, const int N,
                  const int NRHS, double *A, const int lda, double *B, const int ldb);
/* clapack_dgelqf: include/clapack.h:90, interfaces/lapack/C/src/clapack_dgelqf.c */
int clapack_dgelqf(const enum CBLAS_ORDER Order, const int M, const int N, double *A, const int lda,
                   double *TAU);
/* ATL_dormqr: src/lapack/ATL_ormqr.c:24-34 (LWORK < 0: workspace query) */
int ATL_dormqr(const enum CBLAS_SIDE SIDE, const enum CBLAS_TRANSPOSE TRANS, const int M, const int N,
               const int K, double *A, const int lda, const double *TAU, double *C, const int ldc, double *WORK,
               const int LWORK);

/* Fortran 77 calling convention (the reference's interfaces/blas/F77/src and
 * interfaces/lapack/F77/src): every argument by address, characters by their
 * first letter (hidden string lengths are not read), column-major arrays,
 * 1-based IPIV in host memory, INFO through its argument; LWORK = -1 is a
 * workspace query. */
void dgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const double *alpha,
            const double *a, const int *lda, const double *b, const int *ldb, const double *beta, double *c,
            const int *ldc);                                          /* blas/F77/src/dgemm.f */
void sgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const float *alpha,
            const float *a, const int *lda, const float *b, const int *ldb, const float *beta, float *c,
            const int *ldc);                                          /* blas/F77/src/sgemm.f */
void zgemm_(const char *transa, const char *transb, const int *m, const int *n, const int *k, const double *alpha,
            const double *a, const int *lda, const double *b, const int *ldb, const double *beta, double *c,
            const int *ldc);                                          /* blas/F77/src/zgemm.f */
void dtrsm_(const char *side, const char *uplo, const char *transa, const char *diag, const int *m, const int *n,
            const double *alpha, const double *a, const int *lda, double *b, const int *ldb);  /* dtrsm.f */
void dtrmm_(const char *side, const char *uplo, const char *transa, const char *diag, const int *m, const int *n,
            const double *alpha, const double *a, const int *lda, double *b, const int *ldb);  /* dtrmm.f */
void dsyrk_(const char *uplo, const char *trans, const int *n, const int *k, const double *alpha, const double *a,
            const int *lda, const double *beta, double *c, const int *ldc);                   /* dsyrk.f */
void dsymm_(const char *side, const char *uplo, const int *m, const int *n, const double *alpha, const double *a,
            const int *lda, const double *b, const int *ldb, const double *beta, double *c,
            const int *ldc);                                                                  /* dsymm.f */
void dsyr2k_(const char *uplo, const char *trans, const int *n, const int *k, const double *alpha, const double *a,
             const int *lda, const double *b, const int *ldb, const double *beta, double *c,
             const int *ldc);                                                                 /* dsyr2k.f */
void dgetrf_(const int *m, const int *n, double *a, const int *lda, int *ipiv, int *info);  /* lapack/F77/src/dgetrf.f */
void dgetrs_(const char *trans, const int *n, const int *nrhs, const double *a, const int *lda, const int *ipiv,
             double *b, const int *ldb, int *info);                                            /* dgetrs.f */
void dgesv_(const int *n, const int *nrhs, double *a, const int *lda, int *ipiv, double *b, const int *ldb,
            int *info);                                                                        /* dgesv.f */
void dgetri_(const int *n, double *a, const int *lda, const int *ipiv, double *work, const int *lwork,
             int *info);                                                                       /* dgetri.f */
void dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info);           /* dpotrf.f */
void dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda, double *b,
             const int *ldb, int *info);                                                       /* dpotrs.f */
void dposv_(const char *uplo, const int *n, const int *nrhs, double *a, const int *lda, double *b, const int *ldb,
            int *info);                                                                        /* dposv.f */
void dpotri_(const char *uplo, const int *n, double *a, const int *lda, int *info);           /* dpotri.f */
void dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info); /* dtrtri.f */
void dlauum_(const char *uplo, const int *n, double *a, const int *lda, int *info);           /* dlauum.f */
void dgeqrf_(const int *m, const int *n, double *a, const int *lda, double *tau, double *work, const int *lwork,
             int *info);                                                                       /* dgeqrf.f */
void dgelqf_(const int *m, const int *n, double *a, const int *lda, double *tau, double *work, const int *lwork,
             int *info);                                                                       /* dgelqf.f */
void dgels_(const char *trans, const int *m, const int *n, const int *nrhs, double *a, const int *lda, double *b,
            const int *ldb, double *work, const int *lwork, int *info);                        /* dgels.f */

/* cblas_xerbla / cblas_errprn: interfaces/blas/C/src/cblas_xerbla.c:13-28,
 * cblas_errprn.c (error reporting of the drop-in entry points) */
void cblas_xerbla(int p, const char *rout, const char *form, ...);
int cblas_errprn(int ierr, int info, char *form, ...);

/* ---------------------------------------------------------------- Part 2 */

/* Library control.  atlb_init(dev) selects the GPU (-1: keep the default,
 * device 0 or $ATLAS_B200_DEVICE) and returns the device in use.  Error mode
 * 0 = exit(-1) on a bad argument (the reference's behaviour), 1 = return the
 * negative argument position.  Each host thread gets its own stream;
 * atlb_set_stream() substitutes a caller's cudaStream_t (NULL: restore). */
int atlb_init(int device);
void atlb_set_error_mode(int mode);
int atlb_get_error_mode(void);
int atlb_last_error(void);
int atlb_last_cuda_error(void);
void *atlb_get_stream(void);
void atlb_set_stream(void *stream);
int atlb_sync(void);

/* Device-pointer variants: column-major, all pointers in device memory,
 * enqueued on the library stream and NOT synchronised.  Integer arguments
 * use the CBLAS enum values.  Return 0, or -(position) of a bad argument.
 * *dinfo (device) receives the LAPACK info value. */
int atlb_dgemm_dev(int TransA, int TransB, int M, int N, int K, double alpha, const double *A,
                   int lda, const double *B, int ldb, double beta, double *C, int ldc);
int atlb_sgemm_dev(int TransA, int TransB, int M, int N, int K, float alpha, const float *A,
                   int lda, const float *B, int ldb, float beta, float *C, int ldc);
/* FP32 GEMM on the tensor cores: operands rounded to TF32 (prec 1) or BF16
 * (prec 2), or split into TF32 high/low parts whose three products come close
 * to FP32 accuracy (prec 3; the FP32 accumulation of the tensor cores limits
 * it at long K); FP32 accumulation (tcgen05, TMEM accumulators). */
int atlb_sgemm_tc_dev(int prec, int TransA, int TransB, int M, int N, int K, float alpha,
                      const float *A, int lda, const float *B, int ldb, float beta, float *C,
                      int ldc);
int atlb_dtrsm_dev(int Side, int Uplo, int TransA, int Diag, int M, int N, double alpha,
                   const double *A, int lda, double *B, int ldb);
int atlb_dsyrk_dev(int Uplo, int Trans, int N, int K, double alpha, const double *A, int lda,
                   double beta, double *C, int ldc);
/* Tunable driver parameters.  Stand-in for the reference's install-time
 * tuning output (tune/blas/gemm/gmmsearch.c:3604-3634 writes the chosen
 * kernels and blockings into generated headers): atlas_b200/tune.py times the
 * candidates on the GPU and writes tuning.conf beside the library, which is
 * read on first use (ATLAS_B200_TUNE_FILE overrides the path, "none" skips
 * it).  Names: getrf_nb, potrf_nb, dgemm_group, dgemm_splitk, lookahead,
 * mixed_tc_min_work_log2, lookahead_reserve_sms, sgetrf_nb.  get returns
 * INT_MIN for an unknown name; set
 * returns the stored (clamped) value or -1; load returns the number of values
 * read or -1. */
int atlb_tune_get(const char *name);
int atlb_tune_set(const char *name, int value);
int atlb_tune_load(const char *path);
int atlb_tune_count(void);
const char *atlb_tune_name(int i);

/* atlb_dtrsm_dev without any device allocation.  No counterpart in the
 * reference.  For callers that cannot let the library call cudaMalloc:
 * applications whose device memory is owned by their own pool or framework
 * allocator, and programs with a fixed memory budget checked up front.  The
 * workspace is a 2 MiB array compiled into the library (held on every GPU
 * that loads it until exit), so the triangle's order (M for Side = Left, N
 * for Right) may be at most 4096; larger orders are rejected with a message
 * and -5 / -6.  The first call on a device looks up the array's device
 * address (on the library's device, whatever device the calling thread has
 * current); make it before any stream capture starts.  All calls share the
 * array: calls that overlap on the GPU race on it. */
int atlb_dtrsm_dev_noalloc(int Side, int Uplo, int TransA, int Diag, int M, int N, double alpha,
                           const double *A, int lda, double *B, int ldb);
int atlb_dgetrf_dev(int M, int N, double *A, int lda, int *ipiv, int *dinfo);
/* FP32 LU with partial pivoting, the factorization inside the mixed-precision
 * solvers (no counterpart in the reference; LAPACK sgetrf's arguments).
 * Trailing updates in FP32 (prec 0), TF32 (1), BF16 (2) or split TF32 (3).
 * *dinfo: 0 or the first zero pivot (1-based). */
int atlb_sgetrf_dev(int M, int N, float *A, int lda, int *ipiv, int *dinfo, int prec);
int atlb_dgetrs_dev(int Trans, int N, int NRHS, const double *A, int lda, const int *ipiv,
                    double *B, int ldb);
int atlb_dpotrf_dev(int Uplo, int N, double *A, int lda, int *dinfo);
int atlb_dpotrs_dev(int Uplo, int N, int NRHS, const double *A, int lda, double *B, int ldb);
int atlb_dgeqrf_dev(int M, int N, double *A, int lda, double *tau);
/* C = op(Q) C (Side Left) or C op(Q) (Right), Q from atlb_dgeqrf_dev's K
 * reflectors (device pointers, asynchronous; ATL_ormqr's operation). */
int atlb_dormqr_dev(int Side, int Trans, int M, int N, int K, const double *A, int lda, const double *tau,
                    double *C, int ldc);

/* Mixed-precision solvers (no counterpart in the reference; LAPACK's
 * dsgesv/dsposv contract).  Factor an FP32 copy of A on the GPU -- trailing
 * updates in FP32 (prec 0), on the tensor cores in TF32 (1), BF16 with FP32
 * accumulation (2), or near-FP32 split TF32 (3) -- then refine in FP64 until every column reaches a
 * normwise backward error ||b-Ax||_inf/(||A||_inf ||x||_inf + ||b||_inf) <=
 * N*2^-53.  A and B are unchanged and *iter >= 0 (refinement steps) on
 * success; otherwise the FP64 solver runs, A/ipiv hold its factors and *iter
 * < 0 (-3: FP32 factorization broke down, -31: no convergence).  Returns
 * info (0, > 0 singular / not positive definite, < 0 bad argument).  Host or
 * device pointers; synchronous.  Refinement steps are plain (one solve with
 * the low-precision factors) until a step gains less than a digit; from
 * then on -- and from the first step for BF16 (prec 2) -- each step is a
 * GMRES-IR correction: FP64 GMRES on the system preconditioned by the
 * low-precision factors (up to 8 right-hand sides). */
int atlb_dsgesv(int N, int NRHS, double *A, int lda, int *ipiv, double *B, int ldb, double *X,
                int ldx, int prec, int *iter);
int atlb_dsposv(int Uplo, int N, int NRHS, double *A, int lda, double *B, int ldb, double *X,
                int ldx, int prec, int *iter);
/* GMRES steps (Arnoldi vectors) of the calling thread's last mixed solve. */
int atlb_mixed_krylov_steps(void);
/* atlb_dsgesv with a choice of factorization: pivoting 0 = partial pivoting
 * (as atlb_dsgesv), 1 = random butterfly transformation U^T A V of the
 * matrix followed by LU without pivoting (no column-by-column pivot search;
 * the FP64 refinement against the original A restores accuracy, and the FP64
 * fallback covers a failed factorization).  ipiv is only written by the
 * fallback. */
int atlb_dsgesv_ex(int N, int NRHS, double *A, int lda, int *ipiv, double *B, int ldb, double *X,
                   int ldx, int prec, int pivoting, int *iter);

/* Split-integer (Ozaki) DGEMM: C = alpha*op(A)*op(B) + beta*C with FP64
 * operands cut into `slices` (2..12) signed 7-bit digit planes after exact
 * per-row / per-column power-of-two scaling, the digit-plane products run on
 * the INT8 tensor cores with exact INT32 accumulation and are recombined in
 * FP64.  `slices` = 7-8 gives FP64-level accuracy.  No counterpart in the
 * reference.  _dev: device pointers, asynchronous; the other form accepts
 * host or device pointers and is synchronous.  Returns 0 or -(bad argument). */
int atlb_dgemm_ozaki_dev(int TransA, int TransB, int M, int N, int K, double alpha,
                         const double *A, int lda, const double *B, int ldb, double beta,
                         double *C, int ldc, int slices);
int atlb_dgemm_ozaki(int TransA, int TransB, int M, int N, int K, double alpha, const double *A,
                     int lda, const double *B, int ldb, double beta, double *C, int ldc,
                     int slices);

/* Batched, uneven-size problems (no counterpart in the reference).  All
 * pointers inside the arrays are DEVICE pointers; the arrays themselves are
 * host arrays of `count` entries.  Each batch runs as one persistent launch
 * whose CTAs take work (problems, or GEMM tiles) largest first from an atomic
 * counter.  Column-major; returns 0 or -(bad argument).
 *   atlb_dgemm_batched_dev: C[i] = alpha*op(A[i])*op(B[i]) + beta*C[i]; returns
 *     after the launch is enqueued (asynchronous on the library stream).
 *   atlb_dposv_batched: Cholesky (lower triangle) + solve of nrhs[i] right-hand
 *     sides, orders up to 256; info[i] (host) = potrf info; synchronous.
 *   atlb_dgesv_batched: LU with partial pivoting (ipiv[i]: device, 0-based) and,
 *     when B is not NULL, the solve; orders up to 256; synchronous. */
int atlb_dgemm_batched_dev(int TransA, int TransB, int count, const int *M, const int *N,
                           const int *K, double alpha, const double *const *A, const int *lda,
                           const double *const *B, const int *ldb, double beta, double *const *C,
                           const int *ldc);
int atlb_dposv_batched(int count, const int *n, double *const *A, const int *lda, double *const *B,
                       const int *ldb, const int *nrhs, int *info);
/* atlb_dgetrf_batched: the factorization alone (atlb_dgesv_batched with B NULL). */
int atlb_dgetrf_batched(int count, const int *n, double *const *A, const int *lda, int *const *ipiv, int *info);
int atlb_dgesv_batched(int count, const int *n, double *const *A, const int *lda, int *const *ipiv,
                       double *const *B, const int *ldb, const int *nrhs, int *info);

/* Adjoints (reverse-mode derivatives) of the factorizations and solves, for
 * gradient-based callers; no counterpart in the reference.  Device pointers,
 * column-major, asynchronous on the library stream; return 0 or -(bad arg).
 *   atlb_dpotrf_adjoint_dev: A = L L^T (L lower): Abar = (S + S^T)/2 with
 *     S = L^-T Phi(L^T Lbar) L^-1 (Phi: lower triangle, diagonal halved).
 *   atlb_dpotrs_adjoint_dev: X = A^-1 B with A = L L^T: Bbar = A^-1 Xbar and
 *     Abar -= (Bbar X^T + X Bbar^T)/2 (accumulates into Abar).
 *   atlb_dgetrs_adjoint_dev: X = A^-1 B with the getrf factors: Bbar = A^-T Xbar
 *     and Abar -= Bbar X^T (accumulates).
 *   atlb_dgetrf_adjoint_dev: A = P L U: Abar = P L^-T (stril(L^T Lbar) +
 *     triu(Ubar U^T)) U^-T (overwrites Abar). */
int atlb_dpotrf_adjoint_dev(int N, const double *L, int ldl, const double *Lbar, int ldlb,
                            double *Abar, int ldab);
int atlb_dpotrs_adjoint_dev(int N, int NRHS, const double *L, int ldl, const double *X, int ldx,
                            const double *Xbar, int ldxb, double *Bbar, int ldbb, double *Abar,
                            int ldab);
int atlb_dgetrs_adjoint_dev(int N, int NRHS, const double *LU, int ldlu, const int *ipiv,
                            const double *X, int ldx, const double *Xbar, int ldxb, double *Bbar,
                            int ldbb, double *Abar, int ldab);
/* Batched adjoints (no counterpart in the reference): the potrf and potrs
 * adjoints above for `count` independent problems of order n[i] <= 256 in one
 * persistent launch each.  The arrays of device pointers and sizes are host
 * memory, copied before the call returns; the work itself is asynchronous on
 * the library stream.  Return -2 .. -13: the first bad argument position of
 * any problem. */
int atlb_dpotrf_adjoint_batched_dev(int count, const int *n, const double *const *L, const int *ldl,
                                    const double *const *Lbar, const int *ldlb, double *const *Abar,
                                    const int *ldab);
int atlb_dpotrs_adjoint_batched_dev(int count, const int *n, const int *nrhs, const double *const *L,
                                    const int *ldl, const double *const *X, const int *ldx,
                                    const double *const *Xbar, const int *ldxb, double *const *Bbar,
                                    const int *ldbb, double *const *Abar, const int *ldab);
int atlb_dgetrf_adjoint_dev(int N, const double *LU, int ldlu, const int *ipiv, const double *Lbar,
                            int ldlb, const double *Ubar, int ldub, double *Abar, int ldab);

#ifdef __cplusplus
}
#endif
#endif /* ATLAS_B200_H */
