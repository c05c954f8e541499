/* Test infrastructure only (the CPU oracle; never linked by the GPU library).
 *
 * Cache-blocked, multi-threaded level-3 kernels under the oracle's LAPACK
 * restatement, so that the oracle finishes the benchmark-size problems
 * (getrf / getrs at N = 8192) in seconds and can serve as the timed CPU
 * baseline.  They restate the structure of ATLAS's own threaded GEMM -- copy
 * operand blocks into access-major panels (src/blas/ammm/ATL_iploops.c:
 * doAmmBlk), run a register-blocked micro-kernel over them
 * (include/atlas_amm.h: ammkern_t), split the output into blocks among the
 * host threads (src/threads/blas/level3/ATL_tgemm.c:541-628) -- and the
 * recursive triangular solve of src/blas/ulevel3/ATL_trsm.c (halve the
 * triangle, solve, update the rest with GEMM).  Results equal the plain
 * loops' to rounding: sums are taken in a different order.
 *
 * Micro-kernels: 16 x 6 tiles of C, one for AVX-512 (two 8-wide vectors per
 * column) and one for AVX2+FMA (two 8 x 6 halves of 4-wide vectors), chosen
 * at run time; plain C otherwise.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_NOTRANS 111
#define ORC_UPPER 121
#define ORC_LOWER 122
#define ORC_UNIT 132
#define ORC_LEFT 141

#define MR 16
#define NR 6
#define KC 256
#define MC 128          /* multiple of MR */
#define NC 384          /* multiple of NR */

int orc_get_threads(void);

/* ---------------------------------------------------------------- thread pool */
typedef void (*orc_task_fn)(void *ctx, int task);
static struct {
  pthread_mutex_t mu;
  pthread_cond_t go, done;
  int nthreads;           /* workers started (excluding the caller) */
  unsigned long gen;      /* bumps once per dispatched job */
  orc_task_fn fn;
  void *ctx;
  int ntasks;
  int next;               /* next task index (atomic) */
  int busy;               /* workers still inside the current job */
} P = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, PTHREAD_COND_INITIALIZER, 0, 0,
       NULL, NULL, 0, 0, 0};

static void run_tasks(void)
{
  for (;;) {
    int t = __atomic_fetch_add(&P.next, 1, __ATOMIC_RELAXED);
    if (t >= P.ntasks) break;
    P.fn(P.ctx, t);
  }
}

static void *worker(void *arg)
{
  unsigned long seen = 0;
  (void)arg;
  pthread_mutex_lock(&P.mu);
  for (;;) {
    while (P.gen == seen) pthread_cond_wait(&P.go, &P.mu);
    seen = P.gen;
    pthread_mutex_unlock(&P.mu);
    run_tasks();
    pthread_mutex_lock(&P.mu);
    if (--P.busy == 0) pthread_cond_signal(&P.done);
  }
  return NULL;
}

/* Runs fn(ctx, 0..ntasks-1) on the caller plus up to orc_get_threads()-1
 * pool workers (jobs are not nested: a task never dispatches). */
static void par_tasks(int ntasks, orc_task_fn fn, void *ctx)
{
  int want = orc_get_threads() - 1;
  if (want > ntasks - 1) want = ntasks - 1;
  if (want <= 0) {
    for (int t = 0; t < ntasks; t++) fn(ctx, t);
    return;
  }
  pthread_mutex_lock(&P.mu);
  while (P.nthreads < want && P.nthreads < 255) {
    pthread_t th;
    if (pthread_create(&th, NULL, worker, NULL) != 0) break;
    pthread_detach(th);
    P.nthreads++;
  }
  P.fn = fn;
  P.ctx = ctx;
  P.ntasks = ntasks;
  P.next = 0;
  P.busy = P.nthreads;
  P.gen++;
  pthread_cond_broadcast(&P.go);
  pthread_mutex_unlock(&P.mu);
  run_tasks();
  pthread_mutex_lock(&P.mu);
  while (P.busy > 0) pthread_cond_wait(&P.done, &P.mu);
  pthread_mutex_unlock(&P.mu);
}

struct range_job { int n, parts; void (*fn)(void *, int, int); void *ctx; };
static void range_task(void *c, int t)
{
  const struct range_job *r = (const struct range_job *)c;
  const int lo = (int)((int64_t)r->n * t / r->parts), hi = (int)((int64_t)r->n * (t + 1) / r->parts);
  if (hi > lo) r->fn(r->ctx, lo, hi);
}

/* fn(ctx, lo, hi) over one slice of 0..n-1 per host thread */
void orc_pool_ranges(int n, void (*fn)(void *, int, int), void *ctx)
{
  int parts = orc_get_threads();
  if (parts > n) parts = n;
  if (parts <= 1) {
    if (n > 0) fn(ctx, 0, n);
    return;
  }
  struct range_job r = {n, parts, fn, ctx};
  par_tasks(parts, range_task, &r);
}

/* ---------------------------------------------------------------- micro-kernels */
/* Ct (16 x 6, column-major, ld 16) = sum_k Ap[k*16 + 0..15] * Bp[k*6 + 0..5] */
typedef double v8d __attribute__((vector_size(64)));
typedef double v4d __attribute__((vector_size(32)));

__attribute__((target("avx512f")))
static void kern_avx512(int kc, const double *Ap, const double *Bp, double *Ct)
{
  v8d c00 = {0}, c01 = {0}, c02 = {0}, c03 = {0}, c04 = {0}, c05 = {0};
  v8d c10 = {0}, c11 = {0}, c12 = {0}, c13 = {0}, c14 = {0}, c15 = {0};
  for (int k = 0; k < kc; k++) {
    v8d a0, a1;
    memcpy(&a0, Ap + 16 * k, 64);
    memcpy(&a1, Ap + 16 * k + 8, 64);
    const double *b = Bp + 6 * k;
    c00 += a0 * b[0]; c10 += a1 * b[0];
    c01 += a0 * b[1]; c11 += a1 * b[1];
    c02 += a0 * b[2]; c12 += a1 * b[2];
    c03 += a0 * b[3]; c13 += a1 * b[3];
    c04 += a0 * b[4]; c14 += a1 * b[4];
    c05 += a0 * b[5]; c15 += a1 * b[5];
  }
  memcpy(Ct + 0, &c00, 64);  memcpy(Ct + 8, &c10, 64);
  memcpy(Ct + 16, &c01, 64); memcpy(Ct + 24, &c11, 64);
  memcpy(Ct + 32, &c02, 64); memcpy(Ct + 40, &c12, 64);
  memcpy(Ct + 48, &c03, 64); memcpy(Ct + 56, &c13, 64);
  memcpy(Ct + 64, &c04, 64); memcpy(Ct + 72, &c14, 64);
  memcpy(Ct + 80, &c05, 64); memcpy(Ct + 88, &c15, 64);
}

__attribute__((target("avx2,fma")))
static void kern_avx2_half(int kc, const double *Ap, const double *Bp, double *Ct)
{ /* rows 0..7 of the 16-row panel at Ap (Ap already offset for the half) */
  v4d c00 = {0}, c01 = {0}, c02 = {0}, c03 = {0}, c04 = {0}, c05 = {0};
  v4d c10 = {0}, c11 = {0}, c12 = {0}, c13 = {0}, c14 = {0}, c15 = {0};
  for (int k = 0; k < kc; k++) {
    v4d a0, a1;
    memcpy(&a0, Ap + 16 * k, 32);
    memcpy(&a1, Ap + 16 * k + 4, 32);
    const double *b = Bp + 6 * k;
    c00 += a0 * b[0]; c10 += a1 * b[0];
    c01 += a0 * b[1]; c11 += a1 * b[1];
    c02 += a0 * b[2]; c12 += a1 * b[2];
    c03 += a0 * b[3]; c13 += a1 * b[3];
    c04 += a0 * b[4]; c14 += a1 * b[4];
    c05 += a0 * b[5]; c15 += a1 * b[5];
  }
  memcpy(Ct + 0, &c00, 32);  memcpy(Ct + 4, &c10, 32);
  memcpy(Ct + 16, &c01, 32); memcpy(Ct + 20, &c11, 32);
  memcpy(Ct + 32, &c02, 32); memcpy(Ct + 36, &c12, 32);
  memcpy(Ct + 48, &c03, 32); memcpy(Ct + 52, &c13, 32);
  memcpy(Ct + 64, &c04, 32); memcpy(Ct + 68, &c14, 32);
  memcpy(Ct + 80, &c05, 32); memcpy(Ct + 84, &c15, 32);
}

__attribute__((target("avx2,fma")))
static void kern_avx2(int kc, const double *Ap, const double *Bp, double *Ct)
{
  kern_avx2_half(kc, Ap, Bp, Ct);
  kern_avx2_half(kc, Ap + 8, Bp, Ct + 8);
}

static void kern_plain(int kc, const double *Ap, const double *Bp, double *Ct)
{
  double c[NR][MR] = {{0}};
  for (int k = 0; k < kc; k++)
    for (int j = 0; j < NR; j++)
      for (int i = 0; i < MR; i++) c[j][i] += Ap[MR * k + i] * Bp[NR * k + j];
  memcpy(Ct, c, sizeof(c));
}

typedef void (*kern_fn)(int, const double *, const double *, double *);
static kern_fn pick_kernel(void)
{
  static kern_fn k = NULL;
  if (!k) {
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512f")) k = kern_avx512;
    else if (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) k = kern_avx2;
    else k = kern_plain;
  }
  return k;
}

/* ---------------------------------------------------------------- GEMM */
struct gemm_job {
  int ta, tb, M, N, K;
  double alpha, beta;
  const double *A, *B;
  double *C;
  long lda, ldb, ldc;
  int mt, nt;  /* tile grid */
};

static inline double opA(const struct gemm_job *g, int i, int k)
{
  return g->ta == ORC_NOTRANS ? g->A[(size_t)k * g->lda + i] : g->A[(size_t)i * g->lda + k];
}
static inline double opB(const struct gemm_job *g, int k, int j)
{
  return g->tb == ORC_NOTRANS ? g->B[(size_t)j * g->ldb + k] : g->B[(size_t)k * g->ldb + j];
}

static void pack_a(const struct gemm_job *g, int i0, int mc, int k0, int kc, double *Ap)
{
  for (int p = 0; p < mc; p += MR) {
    double *dst = Ap + (size_t)p * kc;
    const int rows = mc - p < MR ? mc - p : MR;
    if (g->ta == ORC_NOTRANS) {
      for (int k = 0; k < kc; k++) {
        const double *src = g->A + (size_t)(k0 + k) * g->lda + i0 + p;
        int r = 0;
        for (; r < rows; r++) dst[MR * k + r] = src[r];
        for (; r < MR; r++) dst[MR * k + r] = 0.0;
      }
    } else {
      for (int r = 0; r < MR; r++) {
        if (r < rows) {
          const double *src = g->A + (size_t)(i0 + p + r) * g->lda + k0;
          for (int k = 0; k < kc; k++) dst[MR * k + r] = src[k];
        } else {
          for (int k = 0; k < kc; k++) dst[MR * k + r] = 0.0;
        }
      }
    }
  }
}

static void pack_b(const struct gemm_job *g, int k0, int kc, int j0, int nc, double *Bp)
{
  for (int q = 0; q < nc; q += NR) {
    double *dst = Bp + (size_t)q * kc;
    const int cols = nc - q < NR ? nc - q : NR;
    for (int c = 0; c < NR; c++) {
      if (c < cols) {
        if (g->tb == ORC_NOTRANS) {
          const double *src = g->B + (size_t)(j0 + q + c) * g->ldb + k0;
          for (int k = 0; k < kc; k++) dst[NR * k + c] = src[k];
        } else {
          for (int k = 0; k < kc; k++) dst[NR * k + c] = opB(g, k0 + k, j0 + q + c);
        }
      } else {
        for (int k = 0; k < kc; k++) dst[NR * k + c] = 0.0;
      }
    }
  }
}

static void gemm_tile(void *ctx, int task)
{
  const struct gemm_job *g = (const struct gemm_job *)ctx;
  const int it = task % g->mt, jt = task / g->mt;
  const int i0 = it * MC, j0 = jt * NC;
  const int mc = g->M - i0 < MC ? g->M - i0 : MC;
  const int nc = g->N - j0 < NC ? g->N - j0 : NC;
  double *Ap = (double *)aligned_alloc(64, sizeof(double) * MC * KC);
  double *Bp = (double *)aligned_alloc(64, sizeof(double) * KC * NC);
  double Ct[MR * NR] __attribute__((aligned(64)));
  kern_fn kern = pick_kernel();
  /* C = beta * C first (beta == 0: overwritten without being read) */
  for (int j = 0; j < nc; j++) {
    double *c = g->C + (size_t)(j0 + j) * g->ldc + i0;
    if (g->beta == 0.0) memset(c, 0, sizeof(double) * mc);
    else if (g->beta != 1.0) for (int i = 0; i < mc; i++) c[i] *= g->beta;
  }
  for (int k0 = 0; k0 < g->K; k0 += KC) {
    const int kc = g->K - k0 < KC ? g->K - k0 : KC;
    pack_b(g, k0, kc, j0, nc, Bp);
    pack_a(g, i0, mc, k0, kc, Ap);
    for (int q = 0; q < nc; q += NR) {
      const int cols = nc - q < NR ? nc - q : NR;
      for (int p = 0; p < mc; p += MR) {
        const int rows = mc - p < MR ? mc - p : MR;
        kern(kc, Ap + (size_t)p * kc, Bp + (size_t)q * kc, Ct);
        for (int c = 0; c < cols; c++) {
          double *dst = g->C + (size_t)(j0 + q + c) * g->ldc + i0 + p;
          for (int r = 0; r < rows; r++) dst[r] += g->alpha * Ct[MR * c + r];
        }
      }
    }
  }
  free(Ap);
  free(Bp);
}

/* C = alpha*op(A)*op(B) + beta*C (beta == 0: C is not read) */
void orc_dgemm_blk(int ta, int tb, int M, int N, int K, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc)
{
  if (M <= 0 || N <= 0) return;
  struct gemm_job g = {ta, tb, M, N, K, alpha, beta, A, B, C, lda, ldb, ldc,
                       (M + MC - 1) / MC, (N + NC - 1) / NC};
  if (K <= 0 || alpha == 0.0) {
    g.K = 0;
    g.alpha = 0.0;
  }
  if ((double)M * N * (g.K > 0 ? g.K : 1) < 2.0e6) {  /* small: waking the pool costs more */
    for (int t = 0; t < g.mt * g.nt; t++) gemm_tile(&g, t);
    return;
  }
  par_tasks(g.mt * g.nt, gemm_tile, &g);
}

/* ---------------------------------------------------------------- TRSM (left side) */
/* element (i, k) of op(T) for the triangle at T */
static inline double tri(const double *T, long ldt, int trans, int i, int k)
{
  return trans == ORC_NOTRANS ? T[(size_t)k * ldt + i] : T[(size_t)i * ldt + k];
}

struct trsm_leaf { const double *T; long ldt; int trans, diag, lower, n, N; double *B; long ldb; };
static void trsm_leaf_cols(void *ctx, int task)
{ /* substitution on a block of up to 64 columns; the triangle is read along
     its stored columns: column sweeps (axpy) for op(T) = T, row sweeps (dot
     products) for op(T) = T^T */
  const struct trsm_leaf *t = (const struct trsm_leaf *)ctx;
  const int c0 = task * 64, c1 = t->N - c0 < 64 ? t->N : c0 + 64;
  const double *T = t->T;
  const long ldt = t->ldt;
  const int n = t->n, unit = t->diag == ORC_UNIT;
  for (int j = c0; j < c1; j++) {
    double *x = t->B + (size_t)j * t->ldb;
    if (t->trans == ORC_NOTRANS) {
      if (t->lower) {
        for (int k = 0; k < n; k++) {
          const double *col = T + (size_t)k * ldt;
          if (!unit) x[k] /= col[k];
          const double xk = x[k];
          for (int i = k + 1; i < n; i++) x[i] -= col[i] * xk;
        }
      } else {
        for (int k = n - 1; k >= 0; k--) {
          const double *col = T + (size_t)k * ldt;
          if (!unit) x[k] /= col[k];
          const double xk = x[k];
          for (int i = 0; i < k; i++) x[i] -= col[i] * xk;
        }
      }
    } else {  /* op(T)(i, k) = T(k, i): row i of op(T) is column i of T */
      if (t->lower) {
        for (int i = 0; i < n; i++) {
          const double *col = T + (size_t)i * ldt;
          double s = x[i];
          for (int k = 0; k < i; k++) s -= col[k] * x[k];
          x[i] = unit ? s : s / col[i];
        }
      } else {
        for (int i = n - 1; i >= 0; i--) {
          const double *col = T + (size_t)i * ldt;
          double s = x[i];
          for (int k = i + 1; k < n; k++) s -= col[k] * x[k];
          x[i] = unit ? s : s / col[i];
        }
      }
    }
  }
}

/* op(T) X = B, X -> B, op(T) of order n lower (lowerEff) or upper */
static void trsm_left_rec(int uplo, int trans, int diag, int n, int N, const double *T, long ldt,
                          double *B, long ldb)
{
  const int lower = (uplo == ORC_LOWER) == (trans == ORC_NOTRANS);
  if (n <= 64) {
    struct trsm_leaf t = {T, ldt, trans, diag, lower, n, N, B, ldb};
    if ((double)n * n * N < 2.0e6)
      for (int c = 0; c < (N + 63) / 64; c++) trsm_leaf_cols(&t, c);
    else
      par_tasks((N + 63) / 64, trsm_leaf_cols, &t);
    return;
  }
  const int n1 = n / 2, n2 = n - n1;
  /* op(T) = [T11 0; T21 T22] (lower) or [T11 T12; 0 T22] (upper), blocks of op(T) */
  const double *T11 = T, *T22 = T + (size_t)n1 * ldt + n1;
  /* the off-diagonal block of op(T): rows n1.. cols 0..n1 (lower) / rows 0..n1 cols n1.. (upper) */
  const double *Toff;
  if (lower) Toff = trans == ORC_NOTRANS ? T + n1 : T + (size_t)n1 * ldt;
  else Toff = trans == ORC_NOTRANS ? T + (size_t)n1 * ldt : T + n1;
  double *B1 = B, *B2 = B + n1;
  if (lower) {
    trsm_left_rec(uplo, trans, diag, n1, N, T11, ldt, B1, ldb);
    orc_dgemm_blk(trans, ORC_NOTRANS, n2, N, n1, -1.0, Toff, (int)ldt, B1, (int)ldb, 1.0, B2, (int)ldb);
    trsm_left_rec(uplo, trans, diag, n2, N, T22, ldt, B2, ldb);
  } else {
    trsm_left_rec(uplo, trans, diag, n2, N, T22, ldt, B2, ldb);
    orc_dgemm_blk(trans, ORC_NOTRANS, n1, N, n2, -1.0, Toff, (int)ldt, B2, (int)ldb, 1.0, B1, (int)ldb);
    trsm_left_rec(uplo, trans, diag, n1, N, T11, ldt, B1, ldb);
  }
}

/* Left-side triangular solve op(T) X = alpha B (X -> B). */
void orc_dtrsm_left_blk(int uplo, int trans, int diag, int M, int N, double alpha, const double *T,
                        int ldt, double *B, int ldb)
{
  if (M <= 0 || N <= 0) return;
  if (alpha != 1.0)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) B[(size_t)j * ldb + i] *= alpha;
  trsm_left_rec(uplo, trans, diag, M, N, T, ldt, B, ldb);
}

/* ---------------------------------------------------------------- row interchanges */
struct laswp_job { int N; double *A; long lda; int k1, k2; const int *ipiv; int inc; };
static void laswp_block(void *ctx, int task)
{ /* the reference's laswp works on 32-column blocks (src/lapack/ATL_laswp.c:7-116) */
  const struct laswp_job *s = (const struct laswp_job *)ctx;
  const int c0 = task * 32, c1 = s->N - c0 < 32 ? s->N : c0 + 32;
  if (s->inc > 0) {
    for (int i = s->k1; i < s->k2; i++) {
      const int ip = s->ipiv[i];
      if (ip == i) continue;
      for (int c = c0; c < c1; c++) {
        double *col = s->A + (size_t)c * s->lda;
        const double t = col[i];
        col[i] = col[ip];
        col[ip] = t;
      }
    }
  } else {
    for (int i = s->k2 - 1; i >= s->k1; i--) {
      const int ip = s->ipiv[i];
      if (ip == i) continue;
      for (int c = c0; c < c1; c++) {
        double *col = s->A + (size_t)c * s->lda;
        const double t = col[i];
        col[i] = col[ip];
        col[ip] = t;
      }
    }
  }
}

void orc_dlaswp_blk(int N, double *A, int lda, int k1, int k2, const int *ipiv, int inc)
{
  if (N <= 0 || k2 <= k1) return;
  struct laswp_job s = {N, A, lda, k1, k2, ipiv, inc};
  par_tasks((N + 31) / 32, laswp_block, &s);
}
