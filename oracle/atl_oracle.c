/*
 * atl_oracle.c -- CPU restatement of ATLAS 3.11.41's dense level-3 BLAS and
 * LAPACK hot path, used ONLY as the correctness checker of the GPU library
 * (tests/, the smoke check and the CPU-baseline leg of bench.py).  Nothing in
 * the shipped library links, loads or calls this file.
 *
 * Everything is column-major FP64 unless stated.  Each routine cites the
 * reference file:line whose behaviour it restates.  The code is written from
 * the algorithms' definitions; only the conventions (pivot rule, sign rule of
 * the Householder reflector, return codes, 0-based ipiv) are kept identical.
 *
 * Pinning: the BLAS part is checked against the reference's own C reference
 * BLAS (src/blas/reference/level3/ATL_dref*.c, compiled unmodified into
 * oracle/_ref/ by oracle/build_ref.sh); the LAPACK part is checked by the
 * residual formulas of the reference's testers (bin/lutst.c, bin/llttst.c,
 * bin/qrtst.c, bin/slvtst.c) and against LAPACK (scipy) conventions in
 * tests/test_oracle.py.  The reference's LAPACK files themselves need headers
 * that only ATLAS's configure step generates (atlas_type.h), so they are not
 * compiled here.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <pthread.h>

/* Host threads used by the loops below (set by orc_set_threads; default 1).
 * A minimal pthread parallel-for, since no OpenMP runtime is present.       */
static int orc_nthreads = 1;
void orc_set_threads(int n) { orc_nthreads = n < 1 ? 1 : n; }
int orc_get_threads(void) { return orc_nthreads; }
typedef void (*orc_range_fn)(void *ctx, int lo, int hi);
/* Splits 0..n-1 into one range per host thread and runs fn on them (the
 * persistent thread pool of orc_fast.c). */
void orc_pool_ranges(int n, orc_range_fn fn, void *ctx);
static void orc_par_for(int n, orc_range_fn fn, void *ctx) { orc_pool_ranges(n, fn, ctx); }

#define ORC_COLMAJOR 102
#define ORC_NOTRANS 111
#define ORC_TRANS 112
#define ORC_UPPER 121
#define ORC_LOWER 122
#define ORC_NONUNIT 131
#define ORC_UNIT 132
#define ORC_LEFT 141
#define ORC_RIGHT 142

#define A_(i, j) A[(size_t)(j) * lda + (i)]
#define B_(i, j) B[(size_t)(j) * ldb + (i)]
#define C_(i, j) C[(size_t)(j) * ldc + (i)]

/* LAPACK's safe minimum (dlamch('S')) and eps (ATL_epsilon returns 2^-52,
 * src/testing/ATL_epsilon.c; ATL_laEPSILON is dlamch('E') = 2^-53). */
static const double ORC_SAFMIN = DBL_MIN;
static const double ORC_LAEPS = 1.1102230246251565e-16;

/* ------------------------------------------------------------------------ */
/* ATL_rand / ATL_srand (src/testing/ATL_rand.c:1-265): a 31-bit LCG
 * x' = (1103515245*x + 12345) mod 2^31 evaluated in two 16/15-bit limbs with
 * 32-bit int wrap-around, seeded through one jump of the same LCG.           */
static int orc_iran[2], orc_ias[2], orc_ics[2];

static int32_t wrap32(int64_t v) { return (int32_t)(uint32_t)(uint64_t)v; }

static void orc_ladd(const int *J, const int *K, int *I)
{ /* ATL_ladd (ATL_rand.c:ladd) */
  int t0 = wrap32((int64_t)K[0] + J[0]), t1;
  t1 = t0 >> 16;
  I[0] = t0 - (t1 << 16);
  t0 = wrap32((int64_t)t1 + K[1] + J[1]);
  I[1] = t0 - ((t0 >> 15) << 15);
}

static void orc_lmul(const int *K, const int *J, int *I)
{ /* ATL_lmul (ATL_rand.c:lmul) */
  const int ipow30 = 1 << 30;
  int kt, lt;
  kt = wrap32((int64_t)K[0] * J[0]);
  if (kt < 0) kt = (kt + ipow30) + ipow30;
  I[0] = kt - ((kt >> 16) << 16);
  lt = wrap32((int64_t)K[0] * J[1] + (int64_t)K[1] * J[0]);
  if (lt < 0) lt = (lt + ipow30) + ipow30;
  kt = wrap32((int64_t)(kt >> 16) + lt);
  if (kt < 0) kt = (kt + ipow30) + ipow30;
  I[1] = kt - ((kt >> 15) << 15);
}

void orc_srand(int iseed)
{ /* ATL_srand (ATL_rand.c:248-258) */
  int mult[2] = {20077, 16838}, iadd[2] = {12345, 0}, jseed[2];
  int j[2];
  jseed[0] = iseed;
  jseed[1] = iseed >> 16;
  /* one jump: iran = jseed*mult + iadd; multiplier/increment unchanged */
  orc_lmul(jseed, mult, j);
  orc_ladd(j, iadd, orc_iran);
  orc_ias[0] = mult[0]; orc_ias[1] = mult[1];
  orc_ics[0] = iadd[0]; orc_ics[1] = iadd[1];
}

int orc_rand(void)
{ /* ATL_rand (ATL_rand.c:260-265) */
  int out0 = orc_iran[0], out1 = orc_iran[1], j[2];
  orc_lmul(orc_iran, orc_ias, j);
  orc_ladd(j, orc_ics, orc_iran);
  return out0 + (out1 << 16);
}

#define ORC_FILLCONST (-2560000000.0)

void orc_gegen(int M, int N, double *A, int lda, int seed)
{ /* ATL_gegen + gefillgap (src/testing/ATL_gegen.c:7-59);
     dumb_rand = 0.5 - rand/2^31 (include/atlas_tst.h:17-18) */
  orc_srand(seed);
  for (int j = 0; j < N; j++) {
    for (int i = M; i < lda; i++) A_(i, j) = ORC_FILLCONST;
  }
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) A_(i, j) = 0.5 - ((double)orc_rand()) / 2147483648.0;
}

int orc_gechkgap(int M, int N, const double *A, int lda)
{ /* ATL_gechkgap (ATL_gegen.c:21-44): count overwrites of the lda gap */
  int bad = 0;
  for (int j = 0; j < N; j++)
    for (int i = M; i < lda; i++)
      if (A_(i, j) != ORC_FILLCONST) bad++;
  return bad;
}

/* ------------------------------------------------------------------------ */
/* Seeded counter-based generators for the benchmark distributions (not in
 * the reference: its testers only use gegen).  splitmix64 of (seed, index).  */
static inline uint64_t splitmix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline double u01(uint64_t seed, uint64_t i)
{ /* (0,1): 53 random bits, offset by half an ulp so log() is finite */
  uint64_t r = splitmix64(seed * 0x632BE59BD9B4E019ull + i);
  return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
void orc_fill_uniform(int64_t n, double *x, uint64_t seed, double lo, double hi)
{
  for (int64_t i = 0; i < n; i++) x[i] = lo + (hi - lo) * u01(seed, (uint64_t)i);
}
void orc_fill_normal(int64_t n, double *x, uint64_t seed)
{ /* Box-Muller on consecutive pairs of counter draws */
  for (int64_t i = 0; i < n; i += 2) {
    double u1 = u01(seed, (uint64_t)i), u2 = u01(seed, (uint64_t)i + 1);
    double r = sqrt(-2.0 * log(u1)), t = 6.283185307179586 * u2;
    x[i] = r * cos(t);
    if (i + 1 < n) x[i + 1] = r * sin(t);
  }
}

/* ------------------------------------------------------------------------ */
/* Level-3 BLAS, restating src/blas/reference/level3/ATL_drefgemm*.c,
 * ATL_dreftrsm*.c, ATL_drefsyrk*.c, ATL_dreftrmm*.c (plain loop orders; the
 * order of the k-sum is increasing k, as in the reference loops).            */
struct gemm_ctx { int TA, TB, M, K; double alpha, beta; const double *A; int lda;
                  const double *B; int ldb; double *C; int ldc; };
static void dgemm_cols(void *p, int j0, int j1)
{
  struct gemm_ctx *g = (struct gemm_ctx *)p;
  const double *A = g->A, *B = g->B; double *C = g->C;
  int lda = g->lda, ldb = g->ldb, ldc = g->ldc;
  for (int j = j0; j < j1; j++) {
    for (int i = 0; i < g->M; i++) {
      double t = 0.0;
      for (int l = 0; l < g->K; l++) {
        double a = (g->TA == ORC_NOTRANS) ? A_(i, l) : A_(l, i);
        double b = (g->TB == ORC_NOTRANS) ? B_(l, j) : B_(j, l);
        t += a * b;
      }
      if (g->beta == 0.0) C_(i, j) = g->alpha * t;
      else C_(i, j) = g->alpha * t + g->beta * C_(i, j);
    }
  }
}
/* cache-blocked, threaded versions (orc_fast.c), used above these sizes */
void orc_dgemm_blk(int ta, int tb, int M, int N, int K, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc);
void orc_dtrsm_left_blk(int uplo, int trans, int diag, int M, int N, double alpha, const double *T,
                        int ldt, double *B, int ldb);
void orc_dlaswp_blk(int N, double *A, int lda, int k1, int k2, const int *ipiv, int inc);
#define ORC_BLK_GEMM_WORK (16.0 * 16.0 * 16.0)

void orc_dgemm(int TA, int TB, int M, int N, int K, double alpha,
               const double *A, int lda, const double *B, int ldb,
               double beta, double *C, int ldc)
{ /* C = alpha*op(A)*op(B) + beta*C; beta == 0 overwrites C without reading */
  if ((double)M * N * K > ORC_BLK_GEMM_WORK) {
    orc_dgemm_blk(TA, TB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return;
  }
  struct gemm_ctx g = {TA, TB, M, K, alpha, beta, A, lda, B, ldb, C, ldc};
  dgemm_cols(&g, 0, N);  /* small: one thread (waking the pool costs more) */
}

struct sgemm_ctx { int TA, TB, M, K; float alpha, beta; const float *A; int lda;
                   const float *B; int ldb; float *C; int ldc; };
static void sgemm_cols(void *p, int j0, int j1)
{
  struct sgemm_ctx *g = (struct sgemm_ctx *)p;
  const float *A = g->A, *B = g->B; float *C = g->C;
  int lda = g->lda, ldb = g->ldb, ldc = g->ldc;
  for (int j = j0; j < j1; j++) {
    for (int i = 0; i < g->M; i++) {
      float t = 0.0f;
      for (int l = 0; l < g->K; l++) {
        float a = (g->TA == ORC_NOTRANS) ? A_(i, l) : A_(l, i);
        float b = (g->TB == ORC_NOTRANS) ? B_(l, j) : B_(j, l);
        t += a * b;
      }
      if (g->beta == 0.0f) C_(i, j) = g->alpha * t;
      else C_(i, j) = g->alpha * t + g->beta * C_(i, j);
    }
  }
}
void orc_sgemm(int TA, int TB, int M, int N, int K, float alpha,
               const float *A, int lda, const float *B, int ldb,
               float beta, float *C, int ldc)
{ /* FP32 version of orc_dgemm (ATL_srefgemm*.c) */
  struct sgemm_ctx g = {TA, TB, M, K, alpha, beta, A, lda, B, ldb, C, ldc};
  orc_par_for(N, sgemm_cols, &g);
}

/* op(T)(i,l) of a triangular matrix with the diagonal convention applied */
static inline double tri_el(const double *A, int lda, int uplo, int trans,
                            int diag, int i, int l)
{
  int r = (trans == ORC_NOTRANS) ? i : l, c = (trans == ORC_NOTRANS) ? l : i;
  if (r == c) return (diag == ORC_UNIT) ? 1.0 : A_(r, c);
  if (uplo == ORC_UPPER) return (r < c) ? A_(r, c) : 0.0;
  return (r > c) ? A_(r, c) : 0.0;
}

struct trsm_ctx { int side, uplo, transa, diag, M, N, lowerEff; double alpha;
                  const double *A; int lda; double *B; int ldb; };
static void trsm_range(void *p, int r0, int r1)
{
  struct trsm_ctx *t_ = (struct trsm_ctx *)p;
  const double *A = t_->A; double *B = t_->B;
  int lda = t_->lda, ldb = t_->ldb, M = t_->M, N = t_->N;
  int uplo = t_->uplo, transa = t_->transa, diag = t_->diag;
  if (t_->side == ORC_LEFT) {
    for (int j = r0; j < r1; j++) { /* column j of B solved independently */
      for (int i = 0; i < M; i++) B_(i, j) *= t_->alpha;
      if (t_->lowerEff) { /* forward substitution */
        for (int i = 0; i < M; i++) {
          double t = B_(i, j);
          for (int l = 0; l < i; l++) t -= tri_el(A, lda, uplo, transa, diag, i, l) * B_(l, j);
          B_(i, j) = (diag == ORC_UNIT) ? t : t / tri_el(A, lda, uplo, transa, diag, i, i);
        }
      } else {
        for (int i = M - 1; i >= 0; i--) {
          double t = B_(i, j);
          for (int l = i + 1; l < M; l++) t -= tri_el(A, lda, uplo, transa, diag, i, l) * B_(l, j);
          B_(i, j) = (diag == ORC_UNIT) ? t : t / tri_el(A, lda, uplo, transa, diag, i, i);
        }
      }
    }
  } else {
    /* X*op(A) = B: row i of X solved independently */
    for (int i = r0; i < r1; i++) {
      for (int j = 0; j < N; j++) B_(i, j) *= t_->alpha;
      if (!t_->lowerEff) { /* op(A) upper: x_j = (b_j - sum_{l<j} x_l a_lj)/a_jj */
        for (int j = 0; j < N; j++) {
          double t = B_(i, j);
          for (int l = 0; l < j; l++) t -= B_(i, l) * tri_el(A, lda, uplo, transa, diag, l, j);
          B_(i, j) = (diag == ORC_UNIT) ? t : t / tri_el(A, lda, uplo, transa, diag, j, j);
        }
      } else {
        for (int j = N - 1; j >= 0; j--) {
          double t = B_(i, j);
          for (int l = j + 1; l < N; l++) t -= B_(i, l) * tri_el(A, lda, uplo, transa, diag, l, j);
          B_(i, j) = (diag == ORC_UNIT) ? t : t / tri_el(A, lda, uplo, transa, diag, j, j);
        }
      }
    }
  }
}
void orc_dtrsm(int side, int uplo, int transa, int diag, int M, int N,
               double alpha, const double *A, int lda, double *B, int ldb)
{ /* solve op(A)*X = alpha*B (Left) or X*op(A) = alpha*B (Right); X -> B.
     ATL_dreftrsm (src/blas/reference/level3/ATL_dreftrsm.c) */
  if (side == ORC_LEFT && (double)M * M * N > ORC_BLK_GEMM_WORK) {
    orc_dtrsm_left_blk(uplo, transa, diag, M, N, alpha, A, lda, B, ldb);
    return;
  }
  struct trsm_ctx t = {side, uplo, transa, diag, M, N,
                       (uplo == ORC_LOWER) == (transa == ORC_NOTRANS), alpha, A, lda, B, ldb};
  const double work = side == ORC_LEFT ? (double)M * M * N : (double)N * N * M;
  if (work <= ORC_BLK_GEMM_WORK) trsm_range(&t, 0, side == ORC_LEFT ? N : M);
  else orc_par_for(side == ORC_LEFT ? N : M, trsm_range, &t);
}

void orc_dtrmm(int side, int uplo, int transa, int diag, int M, int N,
               double alpha, const double *A, int lda, double *B, int ldb)
{ /* B = alpha*op(A)*B or alpha*B*op(A) (ATL_dreftrmm*.c) */
  double *W = (double *)malloc(sizeof(double) * (size_t)M * N);
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      double t = 0.0;
      if (side == ORC_LEFT)
        for (int l = 0; l < M; l++) t += tri_el(A, lda, uplo, transa, diag, i, l) * B_(l, j);
      else
        for (int l = 0; l < N; l++) t += B_(i, l) * tri_el(A, lda, uplo, transa, diag, l, j);
      W[(size_t)j * M + i] = alpha * t;
    }
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) B_(i, j) = W[(size_t)j * M + i];
  free(W);
}

struct syrk_ctx { int uplo, trans, N, K; double alpha, beta; const double *A; int lda;
                  double *C; int ldc; };
static void syrk_cols(void *p, int j0, int j1)
{
  struct syrk_ctx *s = (struct syrk_ctx *)p;
  const double *A = s->A; double *C = s->C; int lda = s->lda, ldc = s->ldc;
  for (int j = j0; j < j1; j++) {
    int i0 = (s->uplo == ORC_UPPER) ? 0 : j, i1 = (s->uplo == ORC_UPPER) ? j + 1 : s->N;
    for (int i = i0; i < i1; i++) {
      double t = 0.0;
      for (int l = 0; l < s->K; l++) {
        double a = (s->trans == ORC_NOTRANS) ? A_(i, l) : A_(l, i);
        double b = (s->trans == ORC_NOTRANS) ? A_(j, l) : A_(l, j);
        t += a * b;
      }
      if (s->beta == 0.0) C_(i, j) = s->alpha * t;
      else C_(i, j) = s->alpha * t + s->beta * C_(i, j);
    }
  }
}
void orc_dsyrk(int uplo, int trans, int N, int K, double alpha,
               const double *A, int lda, double beta, double *C, int ldc)
{ /* C = alpha*op(A)*op(A)^T + beta*C on one triangle (ATL_drefsyrk*.c) */
  struct syrk_ctx s = {uplo, trans, N, K, alpha, beta, A, lda, C, ldc};
  orc_par_for(N, syrk_cols, &s);
}

/* ------------------------------------------------------------------------ */
/* LU.                                                                       */
static int orc_idamax(int n, const double *x)
{ /* cblas_idamax: first index of max |x_i|, 0-based */
  int im = 0;
  double m = -1.0;
  for (int i = 0; i < n; i++) {
    double a = fabs(x[i]);
    if (a > m) { m = a; im = i; }
  }
  return n > 0 ? im : 0;
}

void orc_dlaswp(int N, double *A, int lda, int K1, int K2, const int *ipiv, int inci)
{ /* ATL_laswp (src/lapack/ATL_laswp.c:7-116): for i=K1..K2-1 (or reversed
     when inci<0) swap rows i and ipiv[i] over N columns */
  if (K2 <= K1) return;
  if (N >= 64 && (double)N * (K2 - K1) > 65536.0) {  /* 32-column blocks, as the reference does */
    orc_dlaswp_blk(N, A, lda, K1, K2, ipiv, inci);
    return;
  }
  if (inci > 0) {
    for (int i = K1; i < K2; i++) {
      int ip = ipiv[i];
      if (ip != i)
        for (int j = 0; j < N; j++) { double t = A_(i, j); A_(i, j) = A_(ip, j); A_(ip, j) = t; }
    }
  } else {
    for (int i = K2 - 1; i >= K1; i--) {
      int ip = ipiv[i];
      if (ip != i)
        for (int j = 0; j < N; j++) { double t = A_(i, j); A_(i, j) = A_(ip, j); A_(ip, j) = t; }
    }
  }
}

static int orc_getf2(int M, int N, double *A, int lda, int *ipiv)
{ /* ATL_getf2 (src/lapack/ATL_getf2.c:69-96) with LU1 (:10-62): pivot =
     first max |a|, swap whole panel row, scale by 1/pivot (divide when
     |pivot| < SAFMIN), then rank-1 update of the trailing panel.            */
  int MN = M < N ? M : N, iret = 0;
  if (M < 1 || N < 1) return 0;
  for (int j = 0; j < MN; j++) {
    int ip = j + orc_idamax(M - j, &A_(j, j));
    ipiv[j] = ip;
    double piv = A_(ip, j);
    if (piv != 0.0) {
      if (ip != j)
        for (int c = 0; c < N; c++) { double t = A_(j, c); A_(j, c) = A_(ip, c); A_(ip, c) = t; }
      if (fabs(piv) >= ORC_SAFMIN) {
        double r = 1.0 / piv;
        for (int i = j + 1; i < M; i++) A_(i, j) *= r;
      } else {
        /* The reference's divide branch (ATL_getf2.c:54-59) divides A(j,j)
           repeatedly instead of A(i,j); it is reachable only for |pivot| below
           the FP64 normal range.  The intended column divide is restated. */
        for (int i = j + 1; i < M; i++) A_(i, j) /= piv;
      }
    } else if (!iret) {
      iret = j + 1;
    }
    for (int c = j + 1; c < N; c++) {
      double u = A_(j, c);
      if (u != 0.0)
        for (int i = j + 1; i < M; i++) A_(i, c) -= A_(i, j) * u;
    }
  }
  return iret;
}

#define ORC_L1_ELTS 4096 /* L1C_ELTS: 32 KiB of doubles (generated constant) */

int orc_dgetrf(int M, int N, double *A, int lda, int *ipiv)
{ /* ATL_getrfC (src/lapack/ATL_getrfC.c:242-361): recursive left/right
     halving; leaves are getf2 (M*N <= L1) or the single-column case.  The
     two-column LU2 leaf (:46-136) is the same arithmetic as getf2 on 2
     columns and is folded into getf2 here.                                  */
  int MN = M < N ? M : N, ierr = 0;
  if (MN == 0) return 0;
  if ((size_t)M * N <= ORC_L1_ELTS || MN <= 2) return orc_getf2(M, N, A, lda, ipiv);
  int Nleft = MN >> 1, Nright = N - Nleft, i;
  i = orc_dgetrf(M, Nleft, A, lda, ipiv);
  if (i && !ierr) ierr = i;
  double *Ac = A + (size_t)Nleft * lda, *An = Ac + Nleft;
  orc_dlaswp(Nright, Ac, lda, 0, Nleft, ipiv, 1);
  orc_dtrsm(ORC_LEFT, ORC_LOWER, ORC_NOTRANS, ORC_UNIT, Nleft, Nright, 1.0, A, lda, Ac, lda);
  orc_dgemm(ORC_NOTRANS, ORC_NOTRANS, M - Nleft, Nright, Nleft, -1.0, A + Nleft, lda, Ac, lda,
            1.0, An, lda);
  i = orc_dgetrf(M - Nleft, Nright, An, lda, ipiv + Nleft);
  if (i && !ierr) ierr = i + Nleft;
  for (i = Nleft; i < MN; i++) ipiv[i] += Nleft;
  orc_dlaswp(Nleft, A, lda, Nleft, MN, ipiv, 1);
  return ierr;
}

void orc_dgetrs(int trans, int N, int NRHS, const double *A, int lda,
                const int *ipiv, double *B, int ldb)
{ /* ATL_getrs column-major (src/lapack/ATL_getrs.c:34-50) */
  if (!N || !NRHS) return;
  if (trans == ORC_NOTRANS) {
    orc_dlaswp(NRHS, B, ldb, 0, N, ipiv, 1);
    orc_dtrsm(ORC_LEFT, ORC_LOWER, ORC_NOTRANS, ORC_UNIT, N, NRHS, 1.0, A, lda, B, ldb);
    orc_dtrsm(ORC_LEFT, ORC_UPPER, ORC_NOTRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
  } else {
    orc_dtrsm(ORC_LEFT, ORC_UPPER, ORC_TRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
    orc_dtrsm(ORC_LEFT, ORC_LOWER, ORC_TRANS, ORC_UNIT, N, NRHS, 1.0, A, lda, B, ldb);
    orc_dlaswp(NRHS, B, ldb, 0, N, ipiv, -1);
  }
}

/* ------------------------------------------------------------------------ */
/* Cholesky.                                                                 */
static int orc_potf2(int uplo, int N, double *A, int lda)
{ /* unblocked leaf; same arithmetic as ATL_potrfL_{2,3,4} / potrfU_{2,3,4}
     (src/lapack/ATL_potrfL.c:104-202): returns the first non-positive pivot */
  for (int j = 0; j < N; j++) {
    double d = A_(j, j);
    if (uplo == ORC_LOWER)
      for (int l = 0; l < j; l++) d -= A_(j, l) * A_(j, l);
    else
      for (int l = 0; l < j; l++) d -= A_(l, j) * A_(l, j);
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    A_(j, j) = d;
    for (int i = j + 1; i < N; i++) {
      double t;
      if (uplo == ORC_LOWER) {
        t = A_(i, j);
        for (int l = 0; l < j; l++) t -= A_(i, l) * A_(j, l);
        A_(i, j) = t / d;
      } else {
        t = A_(j, i);
        for (int l = 0; l < j; l++) t -= A_(l, i) * A_(l, j);
        A_(j, i) = t / d;
      }
    }
  }
  return 0;
}

int orc_dpotrf(int uplo, int N, double *A, int lda)
{ /* ATL_potrfL / ATL_potrfU (src/lapack/ATL_potrfL.c:204-263,
     src/lapack/ATL_potrfU.c:199-257): left half, trsm of the off-diagonal
     block, syrk of the trailing block, right half; leaves N <= 4.          */
  if (N <= 4) return orc_potf2(uplo, N, A, lda);
  int Nleft = N >> 1, Nright = N - Nleft, ierr;
  ierr = orc_dpotrf(uplo, Nleft, A, lda);
  if (ierr) return ierr;
  if (uplo == ORC_LOWER) {
    double *Ar = A + Nleft, *An = Ar + (size_t)lda * Nleft;
    orc_dtrsm(ORC_RIGHT, ORC_LOWER, ORC_TRANS, ORC_NONUNIT, Nright, Nleft, 1.0, A, lda, Ar, lda);
    orc_dsyrk(ORC_LOWER, ORC_NOTRANS, Nright, Nleft, -1.0, Ar, lda, 1.0, An, lda);
    ierr = orc_dpotrf(uplo, Nright, An, lda);
  } else {
    double *Ac = A + (size_t)lda * Nleft, *An = Ac + Nleft;
    orc_dtrsm(ORC_LEFT, ORC_UPPER, ORC_TRANS, ORC_NONUNIT, Nleft, Nright, 1.0, A, lda, Ac, lda);
    orc_dsyrk(ORC_UPPER, ORC_TRANS, Nright, Nleft, -1.0, Ac, lda, 1.0, An, lda);
    ierr = orc_dpotrf(uplo, Nright, An, lda);
  }
  return ierr ? ierr + Nleft : 0;
}

void orc_dpotrs(int uplo, int N, int NRHS, const double *A, int lda, double *B, int ldb)
{ /* ATL_potrs column-major (src/lapack/ATL_potrs.c:41-60) */
  if (!N || !NRHS) return;
  if (uplo == ORC_UPPER) {
    orc_dtrsm(ORC_LEFT, ORC_UPPER, ORC_TRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
    orc_dtrsm(ORC_LEFT, ORC_UPPER, ORC_NOTRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
  } else {
    orc_dtrsm(ORC_LEFT, ORC_LOWER, ORC_NOTRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
    orc_dtrsm(ORC_LEFT, ORC_LOWER, ORC_TRANS, ORC_NONUNIT, N, NRHS, 1.0, A, lda, B, ldb);
  }
}

/* ------------------------------------------------------------------------ */
/* QR.                                                                       */
static double orc_dnrm2(int n, const double *x)
{ /* scaled 2-norm (cblas_dnrm2 semantics; avoids overflow/underflow) */
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; i++) {
    if (x[i] != 0.0) {
      double a = fabs(x[i]);
      if (scale < a) { ssq = 1.0 + ssq * (scale / a) * (scale / a); scale = a; }
      else ssq += (a / scale) * (a / scale);
    }
  }
  return scale * sqrt(ssq);
}

static double orc_lapy2(double x, double y)
{ /* sqrt(x^2+y^2) without overflow (ATL_lapy2) */
  double xa = fabs(x), ya = fabs(y), w = xa > ya ? xa : ya, z = xa > ya ? ya : xa;
  if (z == 0.0) return w;
  return w * sqrt(1.0 + (z / w) * (z / w));
}

void orc_dlarfg(int N, double *alpha, double *x, double *tau)
{ /* ATL_larfg (src/lapack/ATL_larfg.c:120-189): beta = -sign(alpha)*
     ||(alpha,x)|| with sign(0)=+, tau = (beta-alpha)/beta,
     x *= 1/(alpha-beta), alpha = beta; rescaling loop when beta < safmin.  */
  if (N < 1) { *tau = 0.0; return; }
  double xnorm = orc_dnrm2(N - 1, x);
  if (xnorm == 0.0) { *tau = 0.0; return; }
  double safmin = ORC_SAFMIN / ORC_LAEPS;
  double betap = orc_lapy2(*alpha, xnorm);
  double beta = (*alpha >= 0) ? -betap : betap;
  if (betap < safmin) {
    double rsafmn = 1.0 / safmin;
    int knt = 0;
    do {
      knt++;
      for (int i = 0; i < N - 1; i++) x[i] *= rsafmn;
      beta *= rsafmn;
      *alpha *= rsafmn;
      betap = fabs(beta);
    } while (betap < safmin && knt < 20);
    xnorm = orc_dnrm2(N - 1, x);
    beta = orc_lapy2(*alpha, xnorm);
    if (*alpha > 0) beta = -beta;
    *tau = (beta - *alpha) / beta;
    double s = 1.0 / (*alpha - beta);
    for (int i = 0; i < N - 1; i++) x[i] *= s;
    *alpha = beta;
    for (int j = 0; j < knt; j++) *alpha *= ORC_SAFMIN;
  } else {
    *tau = (beta - *alpha) / beta;
    double s = 1.0 / (*alpha - beta);
    for (int i = 0; i < N - 1; i++) x[i] *= s;
    *alpha = beta;
  }
}

void orc_dgeqr2(int M, int N, double *A, int lda, double *tau)
{ /* ATL_geqr2 (src/lapack/ATL_geqr2.c:81-144): larfg on column i, then
     apply H(i) = I - tau v v^T (v(0)=1) to A(i:M, i+1:N) via w = A^T v.     */
  int k = M < N ? M : N;
  for (int i = 0; i < k; i++) {
    int t = (i + 1 < M - 1) ? i + 1 : M - 1;
    orc_dlarfg(M - i, &A_(i, i), &A_(t, i), &tau[i]);
    if (i < N - 1 && tau[i] != 0.0) {
      double aii = A_(i, i);
      A_(i, i) = 1.0;
      for (int c = i + 1; c < N; c++) {
        double w = 0.0;
        for (int r = i; r < M; r++) w += A_(r, i) * A_(r, c);
        w *= tau[i];
        for (int r = i; r < M; r++) A_(r, c) -= A_(r, i) * w;
      }
      A_(i, i) = aii;
    }
  }
}

void orc_dlarft(int M, int K, const double *V, int ldv, const double *tau,
                double *T, int ldt)
{ /* ATL_larft Forward/Columnwise (src/lapack/ATL_larft.c:646): upper
     triangular T with H(0)H(1)..H(K-1) = I - V T V^T;
     T(0:i,i) = -tau_i T(0:i,0:i) V(:,0:i)^T v_i, T(i,i) = tau_i.            */
  for (int i = 0; i < K; i++) {
    for (int r = 0; r < i; r++) {
      double s = 0.0; /* (V(:,r))^T v_i with v_i(i)=1 and v_i(<i)=0 */
      s += V[(size_t)r * ldv + i];
      for (int q = i + 1; q < M; q++) s += V[(size_t)r * ldv + q] * V[(size_t)i * ldv + q];
      T[(size_t)i * ldt + r] = -tau[i] * s;
    }
    /* T(0:i,i) = T(0:i,0:i) * T(0:i,i) (upper triangular mat-vec, in place) */
    for (int r = 0; r < i; r++) {
      double s = 0.0;
      for (int q = r; q < i; q++) s += T[(size_t)q * ldt + r] * T[(size_t)i * ldt + q];
      T[(size_t)i * ldt + r] = s;
    }
    T[(size_t)i * ldt + i] = tau[i];
    for (int r = i + 1; r < K; r++) T[(size_t)i * ldt + r] = 0.0;
  }
}

void orc_dlarfb_lt(int M, int N, int K, const double *V, int ldv, const double *T,
                   int ldt, double *C, int ldc)
{ /* ATL_larfb Left/Trans/Forward/Columnwise (src/lapack/ATL_larfb.c:156-240):
     C = (I - V T V^T)^T C = C - V T^T (V^T C), V unit lower trapezoidal.    */
  double *W = (double *)calloc((size_t)K * N, sizeof(double));
  for (int j = 0; j < N; j++)
    for (int p = 0; p < K; p++) {
      double s = C_(p, j);
      for (int r = p + 1; r < M; r++) s += V[(size_t)p * ldv + r] * C_(r, j);
      W[(size_t)j * K + p] = s;
    }
  for (int j = 0; j < N; j++) { /* W = T^T W (T upper => T^T lower) */
    for (int p = K - 1; p >= 0; p--) {
      double s = 0.0;
      for (int q = 0; q <= p; q++) s += T[(size_t)p * ldt + q] * W[(size_t)j * K + q];
      W[(size_t)j * K + p] = s;
    }
  }
  for (int j = 0; j < N; j++)
    for (int r = 0; r < M; r++) {
      double s = 0.0;
      int qmax = r < K - 1 ? r : K - 1;
      for (int q = 0; q <= qmax; q++) {
        double v = (q == r) ? 1.0 : V[(size_t)q * ldv + r];
        s += v * W[(size_t)j * K + q];
      }
      C_(r, j) -= s;
    }
  free(W);
}

int orc_dgeqrf(int M, int N, double *A, int lda, double *tau, int nb)
{ /* ATL_geqrf (src/lapack/ATL_geqrf.c:29-196): nb-wide panels factored and
     their block reflector applied to the columns on the right; the final
     panel (all remaining columns) is factored without building T.  The
     reference's recursive panel ATL_geqrr differs from geqr2 in rounding only. */
  int minMN = M < N ? M : N;
  if (M < 1 || N < 1) return 0;
  if (nb < 1) nb = 32;
  int n = (minMN / nb) * nb;
  if (n == minMN) n -= (nb < minMN ? nb : minMN);
  double *T = (double *)malloc(sizeof(double) * (size_t)nb * nb);
  for (int j = 0; j < n; j += nb) {
    orc_dgeqr2(M - j, nb, &A_(j, j), lda, tau + j);
    if (j + nb < N) {
      orc_dlarft(M - j, nb, &A_(j, j), lda, tau + j, T, nb);
      orc_dlarfb_lt(M - j, N - j - nb, nb, &A_(j, j), lda, T, nb, &A_(j, j + nb), lda);
    }
  }
  orc_dgeqr2(M - n, N - n, &A_(n, n), lda, tau + n);
  free(T);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Norms and the testers' residuals.                                         */
double orc_genrm1(int M, int N, const double *A, int lda)
{ /* ATL_genrm1: max column absolute sum */
  double m = 0.0;
  for (int j = 0; j < N; j++) {
    double s = 0.0;
    for (int i = 0; i < M; i++) s += fabs(A_(i, j));
    if (s > m) m = s;
  }
  return m;
}

double orc_infnrm_vec(int n, const double *x)
{
  double m = 0.0;
  for (int i = 0; i < n; i++) if (fabs(x[i]) > m) m = fabs(x[i]);
  return m;
}

double orc_resid_gemm(int TA, int TB, int M, int N, int K, double alpha,
                      const double *A, int lda, const double *B, int ldb,
                      double beta, const double *C0, int ldc0,
                      const double *Ctst, int ldct)
{ /* bin/l3blastst.c:728-731: ||Ctst - Ctrust||_1 / (max(||A||_1,1)*
     max(||B||_1,1)*max(||Ctrust||_1,1)*eps*max(M,N,K)), eps = 2^-52;
     pass if < 50.  C0 holds the input C; the trusted result is recomputed. */
  double *Ct = (double *)malloc(sizeof(double) * (size_t)M * N);
  for (int j = 0; j < N; j++) for (int i = 0; i < M; i++) Ct[(size_t)j * M + i] = C0[(size_t)j * ldc0 + i];
  orc_dgemm(TA, TB, M, N, K, alpha, A, lda, B, ldb, beta, Ct, M);
  double d = 0.0;
  for (int j = 0; j < N; j++) {
    double s = 0.0;
    for (int i = 0; i < M; i++) s += fabs(Ctst[(size_t)j * ldct + i] - Ct[(size_t)j * M + i]);
    if (s > d) d = s;
  }
  int am = TA == ORC_NOTRANS ? M : K, an = TA == ORC_NOTRANS ? K : M;
  int bm = TB == ORC_NOTRANS ? K : N, bn = TB == ORC_NOTRANS ? N : K;
  double na = orc_genrm1(am, an, A, lda), nb = orc_genrm1(bm, bn, B, ldb);
  double nc = orc_genrm1(M, N, Ct, M);
  free(Ct);
  int mx = M > N ? M : N; if (K > mx) mx = K;
  double den = (na > 1 ? na : 1) * (nb > 1 ? nb : 1) * (nc > 1 ? nc : 1) * DBL_EPSILON * mx;
  return d / den;
}

double orc_resid_lu(int M, int N, const double *A0, int lda0, const double *LU, int ldlu,
                    const int *ipiv)
{ /* bin/lutst.c:199-245: rebuild L*U (ATL_LmulUC), apply the row swaps to a
     copy of A, resid = ||P*A - L*U||_1 / (||A||_1 * eps * min(M,N)).        */
  int MN = M < N ? M : N;
  double *PA = (double *)malloc(sizeof(double) * (size_t)M * N);
  double *R = (double *)malloc(sizeof(double) * (size_t)M * N);
  for (int j = 0; j < N; j++) for (int i = 0; i < M; i++) PA[(size_t)j * M + i] = A0[(size_t)j * lda0 + i];
  double nrmA = orc_genrm1(M, N, PA, M);
  orc_dlaswp(N, PA, M, 0, MN, ipiv, 1);
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      double s = 0.0;
      int kmax = i < j ? i : j; if (kmax > MN - 1) kmax = MN - 1;
      for (int k = 0; k <= kmax; k++) {
        double l = (i == k) ? 1.0 : LU[(size_t)k * ldlu + i];
        s += l * LU[(size_t)j * ldlu + k];
      }
      R[(size_t)j * M + i] = PA[(size_t)j * M + i] - s;
    }
  double r = orc_genrm1(M, N, R, M);
  free(PA); free(R);
  if (nrmA == 0.0 || MN == 0) return r;
  return r / (nrmA * DBL_EPSILON * MN);
}

double orc_resid_llt(int uplo, int N, const double *A0, int lda0, const double *F, int ldf)
{ /* bin/llttst.c:298-350: ||A - L*L^T||_1 / (||A||_1 * eps * N)  (or U^T U) */
  double *R = (double *)malloc(sizeof(double) * (size_t)N * N);
  for (int j = 0; j < N; j++)
    for (int i = 0; i < N; i++) {
      double s = 0.0;
      int kmax = i < j ? i : j;
      for (int k = 0; k <= kmax; k++) {
        if (uplo == ORC_LOWER) s += F[(size_t)k * ldf + i] * F[(size_t)k * ldf + j];
        else s += F[(size_t)i * ldf + k] * F[(size_t)j * ldf + k];
      }
      R[(size_t)j * N + i] = A0[(size_t)j * lda0 + i] - s;
    }
  double r = orc_genrm1(N, N, R, N);
  double *Af = (double *)malloc(sizeof(double) * (size_t)N * N);
  for (int j = 0; j < N; j++) for (int i = 0; i < N; i++) Af[(size_t)j * N + i] = A0[(size_t)j * lda0 + i];
  double nrmA = orc_genrm1(N, N, Af, N);
  free(R); free(Af);
  if (nrmA == 0.0 || N == 0) return r;
  return r / (nrmA * DBL_EPSILON * N);
}

double orc_resid_qr(int M, int N, const double *A0, int lda0, const double *QR, int ldqr,
                    const double *tau)
{ /* bin/qrtst.c:1111-1307: form Q explicitly by applying H(0)..H(k-1) to
     the identity, then ||A - Q*R||_1 / (||A||_1 * eps * min(M,N)).          */
  int k = M < N ? M : N;
  double *Q = (double *)calloc((size_t)M * M, sizeof(double));
  for (int i = 0; i < M; i++) Q[(size_t)i * M + i] = 1.0;
  /* Q = H0 H1 ... H(k-1): apply from the right, Q <- Q H_i */
  for (int i = 0; i < k; i++) {
    if (tau[i] == 0.0) continue;
      for (int r = 0; r < M; r++) {
      double w = Q[(size_t)i * M + r];
      for (int q = i + 1; q < M; q++) w += Q[(size_t)q * M + r] * QR[(size_t)i * ldqr + q];
      w *= tau[i];
      Q[(size_t)i * M + r] -= w;
      for (int q = i + 1; q < M; q++) Q[(size_t)q * M + r] -= w * QR[(size_t)i * ldqr + q];
    }
  }
  double *R = (double *)malloc(sizeof(double) * (size_t)M * N);
  for (int j = 0; j < N; j++)
    for (int r = 0; r < M; r++) {
      double s = 0.0;
      int qmax = j < k - 1 ? j : k - 1;
      for (int q = 0; q <= qmax; q++) s += Q[(size_t)q * M + r] * QR[(size_t)j * ldqr + q];
      R[(size_t)j * M + r] = A0[(size_t)j * lda0 + r] - s;
    }
  double rn = orc_genrm1(M, N, R, M);
  double *Af = (double *)malloc(sizeof(double) * (size_t)M * N);
  for (int j = 0; j < N; j++) for (int i = 0; i < M; i++) Af[(size_t)j * M + i] = A0[(size_t)j * lda0 + i];
  double nrmA = orc_genrm1(M, N, Af, M);
  free(Q); free(R); free(Af);
  if (nrmA == 0.0 || k == 0) return rn;
  return rn / (nrmA * DBL_EPSILON * k);
}

double orc_resid_slv(int N, int NRHS, const double *A, int lda, const double *X, int ldx,
                     const double *Xtrue, int ldxt)
{ /* bin/slvtst.c:419-441: ||x - x_true||_inf / (N * eps * ||A||_1 * ||x||_inf)
     maximised over the right-hand sides.                                    */
  double nrmA = orc_genrm1(N, N, A, lda), worst = 0.0;
  for (int j = 0; j < NRHS; j++) {
    double d = 0.0, xn = 0.0;
    for (int i = 0; i < N; i++) {
      double e = fabs(X[(size_t)j * ldx + i] - Xtrue[(size_t)j * ldxt + i]);
      if (e > d) d = e;
      if (fabs(X[(size_t)j * ldx + i]) > xn) xn = fabs(X[(size_t)j * ldx + i]);
    }
    double r = d / (N * DBL_EPSILON * nrmA * (xn > 0 ? xn : 1.0));
    if (r > worst) worst = r;
  }
  return worst;
}

/* ------------------------------------------------------------------------ */
/* Double-double GEMM (Dekker 1971 TwoProduct via fma; Knuth TwoSum): the
 * oracle for the error of FP64 and split-precision GEMMs.  Returns the hi
 * and lo parts of op(A)*op(B) (alpha=1, beta=0).                            */
static inline void two_sum(double a, double b, double *s, double *e)
{
  double x = a + b, bv = x - a, av = x - bv;
  *s = x;
  *e = (a - av) + (b - bv);
}

void orc_ddgemm(int M, int N, int K, const double *A, int lda, const double *B, int ldb,
                double *Chi, double *Clo, int ldc)
{
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      double sh = 0.0, sl = 0.0;
      for (int l = 0; l < K; l++) {
        double a = A_(i, l), b = B_(l, j);
        double p = a * b, pe = fma(a, b, -p);
        double s, e;
        two_sum(sh, p, &s, &e);
        e += sl + pe;
        two_sum(s, e, &sh, &sl);
      }
      Chi[(size_t)j * ldc + i] = sh;
      Clo[(size_t)j * ldc + i] = sl;
    }
}

double orc_normwise_err_dd(int M, int N, const double *C, int ldc, const double *Chi,
                           const double *Clo, int ldr)
{ /* ||C - (Chi+Clo)||_F / ||Chi+Clo||_F, differences taken in double-double */
  double num = 0.0, den = 0.0;
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      double hi = Chi[(size_t)j * ldr + i], lo = Clo[(size_t)j * ldr + i];
      double d = (C[(size_t)j * ldc + i] - hi) - lo;
      num += d * d;
      den += hi * hi;
    }
  return den > 0 ? sqrt(num / den) : sqrt(num);
}
