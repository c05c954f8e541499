// Triangular solve, triangular multiply and row interchanges.
//
// TRSM follows the reference's recursive method (src/blas/ulevel3/ATL_trsm.c:
// 13-228: halve the triangle, solve one half, GEMM-update the other, solve
// it), down to 64x64 leaves.  The leaves multiply by the inverted diagonal
// blocks (all inverted by one launch per solve), so each leaf is a small
// in-place matrix product over every right-hand side at once.
// Every side/uplo/trans case is reduced to an "effective" forward or backward
// solve T*X = B with T and B addressed through (row, column) strides, so one
// leaf kernel serves all eight cases.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace atlb {

template <>
void gemm_dev<double>(int ta, int tb, int M, int N, int K, double alpha, const double *A, long lda,
                      const double *B, long ldb, double beta, double *C, long ldc,
                      cudaStream_t st, int tri) {
  dgemm_dev(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}
template <>
void gemm_dev<float>(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                     const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                     int tri) {
  sgemm_dev(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}

namespace {

constexpr int LEAF = 64;

// One doubling level of the triangular inverse below: for each pair of
// s x s diagonal blocks (already inverted in sW), the off-diagonal block of
// the inverse of the 2s x 2s block.
template <typename T, int s>
__device__ __forceinline__ void trinv_level(T (*sT)[LEAF + 1], T (*sW)[LEAF + 1], T (*sY)[LEAF + 1],
                                            int lower, int tid) {
  constexpr int per = s / 8;  // outputs per thread: (LEAF / 2s) pairs x s x s / 256
  // Y = T21 W11 (lower) or T12 W22 (upper), stored at the off-diagonal block
#pragma unroll
  for (int q = 0; q < per; q++) {
    const int e = tid + q * 256, p = e / (s * s), rem = e % (s * s), i = rem % s, j = rem / s;
    const int d1 = 2 * p * s, d2 = d1 + s;  // the pair's two diagonal blocks
    T acc = T(0);
    if (lower) {
#pragma unroll
      for (int k = 0; k < s; k++) acc = fma(sT[d2 + i][d1 + k], sW[d1 + k][d1 + j], acc);
      sY[d2 + i][d1 + j] = acc;
    } else {
#pragma unroll
      for (int k = 0; k < s; k++) acc = fma(sT[d1 + i][d2 + k], sW[d2 + k][d2 + j], acc);
      sY[d1 + i][d2 + j] = acc;
    }
  }
  __syncthreads();
  // off-diagonal block of the inverse = -W22 Y (lower) or -W11 Y (upper)
#pragma unroll
  for (int q = 0; q < per; q++) {
    const int e = tid + q * 256, p = e / (s * s), rem = e % (s * s), i = rem % s, j = rem / s;
    const int d1 = 2 * p * s, d2 = d1 + s;
    T acc = T(0);
    if (lower) {
#pragma unroll
      for (int k = 0; k < s; k++) acc = fma(sW[d2 + i][d2 + k], sY[d2 + k][d1 + j], acc);
      sW[d2 + i][d1 + j] = -acc;
    } else {
#pragma unroll
      for (int k = 0; k < s; k++) acc = fma(sW[d1 + i][d1 + k], sY[d1 + k][d2 + j], acc);
      sW[d1 + i][d2 + j] = -acc;
    }
  }
  __syncthreads();
}

// Invert the 64x64 (or smaller, last) diagonal blocks of the effective
// triangle T (T(i,k) = Tp[i*tr + k*tc]) into W: block b is stored dense,
// column-major 64x64 at W + b*64*64, zero outside its triangle (a last block
// smaller than 64 is padded with the identity).  One CTA per block, by
// recursive doubling: the eight 8x8 diagonal blocks are inverted by
// substitution (one thread per column), then the inverse is assembled at
// block sizes 8 -> 16 -> 32 -> 64 from
//   lower:  inv([T11 0; T21 T22]) = [W11 0; -W22 T21 W11  W22]
//   upper:  inv([T11 T12; 0 T22]) = [W11  -W11 T12 W22; 0 W22]
// (two small matrix products per level, all pairs of a level at once).
template <typename T>
__global__ void __launch_bounds__(256)
trinv_kernel(int n, const T *__restrict__ Tp, long tr, long tc, int lower, int unit, T *__restrict__ W) {
  extern __shared__ __align__(16) unsigned char trinv_smem[];
  T(*sT)[LEAF + 1] = reinterpret_cast<T(*)[LEAF + 1]>(trinv_smem);
  T(*sW)[LEAF + 1] = sT + LEAF;
  T(*sY)[LEAF + 1] = sW + LEAF;
  const int b = blockIdx.x, r0 = b * LEAF, nb = min(LEAF, n - r0), tid = threadIdx.x;
  const T *Tb = Tp + r0 * tr + r0 * tc;
  {
    T tv[LEAF * LEAF / 256];  // unrolled: all loads of a thread in flight at once
#pragma unroll
    for (int q = 0; q < LEAF * LEAF / 256; q++) {
      const int idx = tid + 256 * q;
      int i, k;
      if (tr == 1) { i = idx % LEAF; k = idx / LEAF; } else { k = idx % LEAF; i = idx / LEAF; }
      T v;
      if (i < nb && k < nb) {
        const bool in_tri = lower ? i > k : i < k;
        v = (i == k) ? (unit ? T(1) : Tb[i * tr + k * tc]) : (in_tri ? Tb[i * tr + k * tc] : T(0));
      } else {
        v = (i == k) ? T(1) : T(0);
      }
      tv[q] = v;
    }
#pragma unroll
    for (int q = 0; q < LEAF * LEAF / 256; q++) {
      const int idx = tid + 256 * q;
      int i, k;
      if (tr == 1) { i = idx % LEAF; k = idx / LEAF; } else { k = idx % LEAF; i = idx / LEAF; }
      sT[i][k] = tv[q];
      sW[i][k] = T(0);
    }
  }
  __syncthreads();
  // 8x8 diagonal blocks: thread (blk, c) solves for column c of block blk
  if (tid < LEAF) {
    const int base = (tid >> 3) * 8, c = tid & 7;
    T x[8];
    if (lower) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        T s = (k == c) ? T(1) : T(0);
#pragma unroll
        for (int m = 0; m < k; m++) s = fma(-sT[base + k][base + m], x[m], s);
        x[k] = s / sT[base + k][base + k];
      }
    } else {
#pragma unroll
      for (int k = 7; k >= 0; k--) {
        T s = (k == c) ? T(1) : T(0);
#pragma unroll
        for (int m = k + 1; m < 8; m++) s = fma(-sT[base + k][base + m], x[m], s);
        x[k] = s / sT[base + k][base + k];
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) sW[base + k][base + c] = x[k];
  }
  __syncthreads();
  trinv_level<T, 8>(sT, sW, sY, lower, tid);
  trinv_level<T, 16>(sT, sW, sY, lower, tid);
  trinv_level<T, 32>(sT, sW, sY, lower, tid);
  T *Wb = W + (long)b * LEAF * LEAF;
#pragma unroll
  for (int q = 0; q < LEAF * LEAF / 256; q++) {
    const int idx = tid + 256 * q;
    Wb[idx] = sW[idx % LEAF][idx / LEAF];
  }
}

// B_blk (nb x m, effective strides) = W_b (nb x nb) * B_blk, in place: one
// CTA per 64-column tile holds W_b and its tile in shared memory.
template <typename T>
__global__ void __launch_bounds__(256)
tri_apply_kernel(int nb, int m, const T *__restrict__ Wb, T *__restrict__ Bp, long br, long bc) {
  extern __shared__ __align__(16) unsigned char tri_smem[];
  T(*sW)[LEAF + 1] = reinterpret_cast<T(*)[LEAF + 1]>(tri_smem);
  T(*sB)[LEAF + 1] = sW + LEAF;
  const int j0 = blockIdx.x * LEAF, tid = threadIdx.x;
  const int mcols = min(LEAF, m - j0);
  // fixed trip counts, unrolled: all 32 loads of a thread are in flight at once
  T wv[LEAF * LEAF / 256], bv[LEAF * LEAF / 256];
#pragma unroll
  for (int q = 0; q < LEAF * LEAF / 256; q++) {
    const int idx = tid + 256 * q, i = idx % LEAF, k = idx / LEAF;
    wv[q] = (i < nb && k < nb) ? Wb[i + (long)k * LEAF] : T(0);
  }
#pragma unroll
  for (int q = 0; q < LEAF * LEAF / 256; q++) {
    const int idx = tid + 256 * q;
    int i, j;
    if (br == 1) { i = idx % LEAF; j = idx / LEAF; } else { j = idx % LEAF; i = idx / LEAF; }
    bv[q] = (i < nb && j < mcols) ? Bp[i * br + (long)(j0 + j) * bc] : T(0);
  }
#pragma unroll
  for (int q = 0; q < LEAF * LEAF / 256; q++) {
    const int idx = tid + 256 * q;
    sW[idx % LEAF][idx / LEAF] = wv[q];
    int i, j;
    if (br == 1) { i = idx % LEAF; j = idx / LEAF; } else { j = idx % LEAF; i = idx / LEAF; }
    sB[i][j] = bv[q];
  }
  __syncthreads();
  const int r = tid % LEAF, cg = tid / LEAF;  // 4 column groups
  T acc[16];
#pragma unroll
  for (int q = 0; q < 16; q++) acc[q] = T(0);
#pragma unroll 8
  for (int k = 0; k < LEAF; k++) {
    const T w = sW[r][k];
#pragma unroll
    for (int q = 0; q < 16; q++) acc[q] = fma(w, sB[k][cg + 4 * q], acc[q]);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 16; q++) sB[r][cg + 4 * q] = acc[q];
  __syncthreads();
  for (int idx = tid; idx < nb * mcols; idx += 256) {
    int i, j;
    if (br == 1) { i = idx % nb; j = idx / nb; } else { j = idx % mcols; i = idx / mcols; }
    Bp[i * br + (long)(j0 + j) * bc] = sB[i][j];
  }
}

template <typename T>
__global__ void scale_strided_kernel(int n, int m, T alpha, T *B, long br, long bc) {
  long total = (long)n * m;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i, j;
    if (br == 1) { i = (int)(idx % n); j = (int)(idx / n); } else { j = (int)(idx % m); i = (int)(idx / m); }
    B[i * br + (long)j * bc] *= alpha;
  }
}

template <typename T>
struct Eff {  // effective problem T*X = B
  const T *Tp; long tr, tc;
  T *Bp; long br, bc;
  int lower, unit;
  const T *W;   // inverted 64x64 diagonal blocks (trinv_kernel)
};

template <typename T>
void gemm_call(SgemmFn fn, int ta, int tb, int M, int N, int K, T alpha, const T *A, long lda,
               const T *B, long ldb, T beta, T *C, long ldc, cudaStream_t st);
template <>
void gemm_call<double>(SgemmFn, int ta, int tb, int M, int N, int K, double alpha,
                       const double *A, long lda, const double *B, long ldb, double beta,
                       double *C, long ldc, cudaStream_t st) {
  dgemm_dev(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, 0);
}
template <>
void gemm_call<float>(SgemmFn fn, int ta, int tb, int M, int N, int K, float alpha,
                      const float *A, long lda, const float *B, long ldb, float beta, float *C,
                      long ldc, cudaStream_t st) {
  (fn ? fn : sgemm_dev)(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, 0);
}

// C (M x N) -= op(A) (M x K) op(B) (K x N) for K <= 64: the product that
// couples the two halves of a TRSM of order <= 128 (the Cholesky's block
// columns).  The general GEMMs pay their K-loop pipeline, or a split-K pass
// with its reduction, for what is one 64-deep step; here a CTA takes a
// 64 x 64 tile of C, copies its slices of op(A) and op(B) into shared memory
// (cp.async, all in flight at once) while its threads load their old C
// values, and each thread computes 4 rows (16 apart) x 4 columns (16 apart).
constexpr int SK_T = 64, SK_K = 64;
template <typename T, bool TA, bool TB>
__global__ void __launch_bounds__(256, 2)
gemm_smallk_kernel(int M, int N, int K, const T *__restrict__ A, long lda, const T *__restrict__ B, long ldb,
                   T *__restrict__ C, long ldc) {
  extern __shared__ __align__(16) unsigned char sk_smem[];
  T(*sA)[SK_T + 1] = reinterpret_cast<T(*)[SK_T + 1]>(sk_smem);  // sA[k][m]
  T(*sB)[SK_T + 1] = sA + SK_K;                                   // sB[k][n]
  const int tid = threadIdx.x, m0 = blockIdx.x * SK_T, n0 = blockIdx.y * SK_T;
  const int tr = tid % 16, tc = tid / 16;
  for (int e = tid; e < SK_K * SK_T; e += 256) {
    // op(A)(m, k) = TA ? A[k + m lda] : A[m + k lda]; the faster index runs along memory
    const int i = TA ? e % SK_K : e / SK_T, r = TA ? e / SK_K : e % SK_T;  // (k, m)
    const bool okA = i < K && m0 + r < M;
    const T *ga = TA ? A + i + (long)(m0 + r) * lda : A + (m0 + r) + (long)i * lda;
    if (sizeof(T) == 8) cp_async8(&sA[i][r], okA ? ga : A, okA);
    else cp_async4(&sA[i][r], okA ? ga : A, okA);
    // op(B)(k, n) = TB ? B[n + k ldb] : B[k + n ldb]
    const int kb = TB ? e / SK_T : e % SK_K, c = TB ? e % SK_T : e / SK_K;
    const bool okB = kb < K && n0 + c < N;
    const T *gb = TB ? B + (n0 + c) + (long)kb * ldb : B + kb + (long)(n0 + c) * ldb;
    if (sizeof(T) == 8) cp_async8(&sB[kb][c], okB ? gb : B, okB);
    else cp_async4(&sB[kb][c], okB ? gb : B, okB);
  }
  cp_async_commit();
  T old[4][4], acc[4][4];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int r = m0 + tr + 16 * a, c = n0 + tc + 16 * q;
      old[a][q] = (r < M && c < N) ? C[r + (long)c * ldc] : T(0);
      acc[a][q] = T(0);
    }
  cp_async_wait<0>();
  __syncthreads();
  for (int i = 0; i < K; i++) {
    T av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; a++) av[a] = sA[i][tr + 16 * a];
#pragma unroll
    for (int q = 0; q < 4; q++) bv[q] = sB[i][tc + 16 * q];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[a][q] = fma(av[a], bv[q], acc[a][q]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int a = 0; a < 4; a++) {
      const int r = m0 + tr + 16 * a, c = n0 + tc + 16 * q;
      if (r < M && c < N) C[r + (long)c * ldc] = old[a][q] - acc[a][q];
    }
}

template <typename T, bool TA, bool TB>
void smallk_launch(int M, int N, int K, const T *A, long lda, const T *B, long ldb, T *C, long ldc, cudaStream_t st) {
  constexpr int smem = 2 * SK_K * (SK_T + 1) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(gemm_smallk_kernel<T, TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem));
    configured = true;
  }
  gemm_smallk_kernel<T, TA, TB><<<dim3(cdiv(M, SK_T), cdiv(N, SK_T)), 256, smem, st>>>(M, N, K, A, lda, B, ldb, C,
                                                                                      ldc);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void gemm_smallk(int ta, int tb, int M, int N, int K, const T *A, long lda, const T *B, long ldb, T *C, long ldc,
                 cudaStream_t st) {
  if (ta == kNoTrans && tb == kNoTrans) smallk_launch<T, false, false>(M, N, K, A, lda, B, ldb, C, ldc, st);
  else if (ta == kNoTrans) smallk_launch<T, false, true>(M, N, K, A, lda, B, ldb, C, ldc, st);
  else if (tb == kNoTrans) smallk_launch<T, true, false>(M, N, K, A, lda, B, ldb, C, ldc, st);
  else smallk_launch<T, true, true>(M, N, K, A, lda, B, ldb, C, ldc, st);
}

// B2 (n2 x m) -= T21 (n2 x n1) * X1 (n1 x m), everything in effective strides.
template <typename T>
void eff_update(const Eff<T> &e, int r2, int n2, int r1, int n1, int m, SgemmFn fn,
                cudaStream_t st) {
  const T *T21 = e.Tp + r2 * e.tr + r1 * e.tc;
  T *B2 = e.Bp + r2 * e.br;
  const T *X1 = e.Bp + r1 * e.br;
  const bool small = n1 <= SK_K && n2 <= 2 * SK_T;  // the coupling product of an order <= 128 solve
  if (e.br == 1) {  // B column-major (ld = bc)
    int ta = (e.tr == 1) ? kNoTrans : kTrans;
    long ldt = (e.tr == 1) ? e.tc : e.tr;
    if (small) gemm_smallk<T>(ta, kNoTrans, n2, m, n1, T21, ldt, X1, e.bc, B2, e.bc, st);
    else gemm_call<T>(fn, ta, kNoTrans, n2, m, n1, T(-1), T21, ldt, X1, e.bc, T(1), B2, e.bc, st);
  } else {  // B^T column-major (m x n) with ld = br: B2^T -= X1^T * T21^T
    int tb = (e.tc == 1) ? kNoTrans : kTrans;
    long ldt = (e.tc == 1) ? e.tr : e.tc;
    if (small) gemm_smallk<T>(kNoTrans, tb, m, n2, n1, X1, e.br, T21, ldt, B2, e.br, st);
    else gemm_call<T>(fn, kNoTrans, tb, m, n2, n1, T(-1), X1, e.br, T21, ldt, T(1), B2, e.br, st);
  }
}

template <typename T>
void eff_solve(const Eff<T> &e, int r0, int n, int m, SgemmFn fn, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  if (n <= LEAF) {
    constexpr int smem = 2 * LEAF * (LEAF + 1) * (int)sizeof(T);
    static bool configured = false;
    if (!configured) {
      ATLB_CUDA_CHECK(cudaFuncSetAttribute(tri_apply_kernel<T>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      configured = true;
    }
    tri_apply_kernel<T><<<cdiv(m, LEAF), 256, smem, st>>>(
        n, m, e.W + (long)(r0 / LEAF) * LEAF * LEAF, e.Bp + r0 * e.br, e.br, e.bc);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  int n1 = std::max(LEAF, (n / 2) / LEAF * LEAF), n2 = n - n1;
  if (e.lower) {
    eff_solve(e, r0, n1, m, fn, st);
    eff_update(e, r0 + n1, n2, r0, n1, m, fn, st);
    eff_solve(e, r0 + n1, n2, m, fn, st);
  } else {
    eff_solve(e, r0 + n1, n2, m, fn, st);
    eff_update(e, r0, n1, r0 + n1, n2, m, fn, st);
    eff_solve(e, r0, n1, m, fn, st);
  }
}

// Row interchanges.  The swaps k1..k2-1 of one call (at most LSW_MAXP of
// them; longer ranges are split) are first reduced to their net effect by one
// CTA: a permutation of the rows [k1, hi) simulated in shared memory, then
// compacted into the list of (destination, source) row moves.  The apply
// kernel then moves only those rows, in parallel over columns (up to 16 per
// CTA): all sources are read into shared memory before any destination is
// written, so the in-place permutation needs no ordering.
constexpr int LSW_MAXP = 256;               // pivots per plan
constexpr int LSW_SPAN = 24576;             // rows the sequential plan can track in shared memory
constexpr int LSW_COLS = 16;

// The plan without a sequential replay, for chunks whose pivots all lie at or
// below their own row (ipiv[k] >= k, as getrf's are); returns false (every
// thread) when the chunk has another pivot, for the replay below.
// With the swaps applied in order k1, k1+1, .., position k's content is final
// after swap k, and a position p is touched again only by swaps j with
// ipiv[j] = p.  Let arr(k) be the row whose content stands at position k just
// before swap k: arr(k) = arr(j) for the last j < k with ipiv[j] = k, and the
// row k itself when there is none.  Then position k ends with arr(k) when
// ipiv[k] = k, else with arr(j) for the last j < k with ipiv[j] = ipiv[k]
// (or row ipiv[k] itself when there is none); a pivot row p >= k2 ends with
// arr(j) for the last j with ipiv[j] = p.  The (pivot row, step) pairs are
// sorted (bitonic, 256 keys) so that "the last j before" is the neighbour in
// sorted order, and arr() follows its chain of earlier steps by pointer
// jumping (8 rounds cover 256 steps).  Applied in the reverse order (inc < 0)
// the swaps give the inverse permutation: each (destination, source) pair is
// reversed.
__device__ bool laswp_plan_parallel(int k1, int k2, const int *__restrict__ ipiv, int inc, int *__restrict__ moves,
                                    int *__restrict__ nmoves, int *__restrict__ ok, int *s_back) {
  __shared__ unsigned long long skey[LSW_MAXP];
  __shared__ int sparent[LSW_MAXP], sprev[LSW_MAXP], sptr[2][LSW_MAXP], sdisp[LSW_MAXP], swsum[LSW_MAXP / 32];
  const int tid = threadIdx.x, nk = k2 - k1, lane = tid & 31, wid = tid >> 5;
  int myp = 0;
  if (tid < LSW_MAXP) {
    if (tid < nk) {
      myp = ipiv[k1 + tid];
      if (myp < k1 + tid) *s_back = 1;
      skey[tid] = ((unsigned long long)(unsigned)myp << 16) | (unsigned)tid;
    } else {
      skey[tid] = ~0ull;
    }
    sparent[tid] = -1;
    sprev[tid] = -1;
  }
  __syncthreads();
  if (*s_back) return false;
  for (int size = 2; size <= LSW_MAXP; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (tid < LSW_MAXP) {
        const int partner = tid ^ stride;
        if (partner > tid) {
          const bool asc = (tid & size) == 0;
          const unsigned long long a = skey[tid], b = skey[partner];
          if ((a > b) == asc) { skey[tid] = b; skey[partner] = a; }
        }
      }
      __syncthreads();
    }
  if (tid < nk) {  // sorted position tid
    const unsigned long long key = skey[tid];
    const int p = (int)(key >> 16), j = (int)(key & 0xffffu), pl = p - k1;
    const bool next_same = tid + 1 < nk && (int)(skey[tid + 1] >> 16) == p;
    if (tid > 0 && (int)(skey[tid - 1] >> 16) == p) sprev[j] = (int)(skey[tid - 1] & 0xffffu);
    // the last step before pl that brought something to position pl
    if (p < k2 && j < pl && (!next_same || (int)(skey[tid + 1] & 0xffffu) == pl)) sparent[pl] = j;
    sdisp[tid] = p >= k2 && !next_same;  // the last swap with pivot row p, below the chunk
  } else if (tid < LSW_MAXP) {
    sdisp[tid] = 0;
  }
  __syncthreads();
  if (tid < nk) sptr[0][tid] = sparent[tid] >= 0 ? sparent[tid] : tid;
  __syncthreads();
  int cur = 0;
#pragma unroll 1
  for (int r = 0; r < 8; r++) {
    if (tid < nk) sptr[cur ^ 1][tid] = sptr[cur][sptr[cur][tid]];
    __syncthreads();
    cur ^= 1;
  }
  // position k1 + tid ends with row fin; the displaced row of sorted position tid
  int fin = 0, dsrc = 0, ddst = 0;
  bool fa = false, fb = false;
  if (tid < nk) {
    const int sv = myp == k1 + tid ? sptr[cur][tid] : sprev[tid];
    fin = sv >= 0 ? k1 + sptr[cur][sv] : myp;
    fa = fin != k1 + tid;
    fb = sdisp[tid] != 0;
    if (fb) {
      const unsigned long long key = skey[tid];
      ddst = (int)(key >> 16);
      dsrc = k1 + sptr[cur][(int)(key & 0xffffu)];
    }
  }
  // destinations in order: the chunk's rows, then the rows below it (block-wide prefix count)
  const int v = (fa ? 1 : 0) | (fb ? 1 << 16 : 0);
  int isc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, isc, o);
    if (lane >= o) isc += u;
  }
  if (lane == 31 && wid < LSW_MAXP / 32) swsum[wid] = isc;
  __syncthreads();
  if (tid < LSW_MAXP) {
    int off = 0, tot = 0;
    for (int w = 0; w < LSW_MAXP / 32; w++) {
      if (w < wid) off += swsum[w];
      tot += swsum[w];
    }
    const int ex = off + isc - v, tota = tot & 0xffff;
    if (fa) {
      const int slot = ex & 0xffff;
      moves[2 * slot] = inc > 0 ? k1 + tid : fin;
      moves[2 * slot + 1] = inc > 0 ? fin : k1 + tid;
    }
    if (fb) {
      const int slot = tota + (ex >> 16);
      moves[2 * slot] = inc > 0 ? ddst : dsrc;
      moves[2 * slot + 1] = inc > 0 ? dsrc : ddst;
    }
    if (tid == 0) { *nmoves = tota + (tot >> 16); *ok = 1; }
  }
  return true;
}

__global__ void __launch_bounds__(1024)
laswp_plan_kernel(int k1, int k2, const int *__restrict__ ipiv, int inc, int *__restrict__ moves,
                  int *__restrict__ nmoves, int *__restrict__ ok) {
  extern __shared__ int perm[];  // LSW_SPAN entries
  __shared__ int s_hi, s_cnt, s_back;
  const int tid = threadIdx.x;
  if (tid == 0) { s_hi = k2; s_cnt = 0; s_back = 0; }
  __syncthreads();
  if (laswp_plan_parallel(k1, k2, ipiv, inc, moves, nmoves, ok, &s_back)) return;
  for (int k = k1 + tid; k < k2; k += blockDim.x) atomicMax(&s_hi, ipiv[k] + 1);
  __syncthreads();
  const int span = s_hi - k1;
  if (span > LSW_SPAN) {  // rows too far apart for the plan: caller falls back
    if (tid == 0) { *ok = 0; *nmoves = 0; }
    return;
  }
  for (int r = tid; r < span; r += blockDim.x) perm[r] = k1 + r;
  __syncthreads();
  if (tid == 0) {
    if (inc > 0) {
      for (int k = k1; k < k2; k++) {
        const int a = k - k1, b = ipiv[k] - k1;
        const int t = perm[a]; perm[a] = perm[b]; perm[b] = t;
      }
    } else {
      for (int k = k2 - 1; k >= k1; k--) {
        const int a = k - k1, b = ipiv[k] - k1;
        const int t = perm[a]; perm[a] = perm[b]; perm[b] = t;
      }
    }
  }
  __syncthreads();
  // the moves in increasing destination order (a block-wide prefix count), so
  // that the apply kernel's neighbouring threads touch neighbouring rows
  __shared__ int s_wsum[32];
  const int chunk = (span + blockDim.x - 1) / blockDim.x, rbeg = tid * chunk, rend = min(span, rbeg + chunk);
  int cnt = 0;
  for (int r = rbeg; r < rend; r++) cnt += perm[r] != k1 + r;
  const int lane = tid & 31, wid = tid >> 5;
  int isc = cnt;  // inclusive scan within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, isc, o);
    if (lane >= o) isc += v;
  }
  if (lane == 31) s_wsum[wid] = isc;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x / 32;
    int w = lane < nw ? s_wsum[lane] : 0, wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += v;
    }
    if (lane < nw) s_wsum[lane] = wi - w;  // exclusive warp offsets
    if (lane == nw - 1) s_cnt = wi;
  }
  __syncthreads();
  int slot = s_wsum[wid] + isc - cnt;
  for (int r = rbeg; r < rend; r++) {
    if (perm[r] != k1 + r) {
      moves[2 * slot] = k1 + r;       // destination row
      moves[2 * slot + 1] = perm[r];  // source row
      slot++;
    }
  }
  __syncthreads();
  if (tid == 0) { *nmoves = s_cnt; *ok = 1; }
}

// One CTA per `cpc` columns (at most LSW_COLS): the move list first comes
// into shared memory, then every thread gathers its sources eight loads at a
// time (independent loads in flight instead of one dependent round trip per
// element), and after one barrier writes them to their destinations.  When
// the plan could not track the rows (*ok == 0), the CTA's first threads
// replay the swaps sequentially on its columns instead, one thread per column.
template <typename T>
__global__ void __launch_bounds__(256)
laswp_apply_kernel(int ncols, int cpc, T *A, long lda, const int *__restrict__ moves,
                   const int *__restrict__ nmoves, const int *__restrict__ ok, int k1, int k2,
                   const int *__restrict__ ipiv, int inc) {
  extern __shared__ __align__(16) unsigned char lsw_smem[];
  T *buf = reinterpret_cast<T *>(lsw_smem);                        // [2*LSW_MAXP][LSW_COLS]
  int *smv = reinterpret_cast<int *>(buf + 2 * LSW_MAXP * LSW_COLS);  // [2*LSW_MAXP][2]
  const int c0 = blockIdx.x * cpc, tid = threadIdx.x;
  const int nc = min(cpc, ncols - c0);
  if (!*ok) {
    if (tid >= nc) return;
    T *col = A + (long)(c0 + tid) * lda;
    if (inc > 0) {
      for (int k = k1; k < k2; k++) {
        const int p = ipiv[k];
        if (p != k) { T t = col[k]; col[k] = col[p]; col[p] = t; }
      }
    } else {
      for (int k = k2 - 1; k >= k1; k--) {
        const int p = ipiv[k];
        if (p != k) { T t = col[k]; col[k] = col[p]; col[p] = t; }
      }
    }
    return;
  }
  const int nm = *nmoves;
  for (int i = tid; i < 2 * nm; i += 256) smv[i] = moves[i];
  __syncthreads();
  // moves fastest: neighbouring threads take neighbouring (sorted) rows of one column
  const int total = nm * nc;
  for (int base = tid; base < total; base += 8 * 256) {
    T v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int idx = base + 256 * q;
      if (idx < total) {
        const int m = idx % nm, c = idx / nm;
        v[q] = A[smv[2 * m + 1] + (long)(c0 + c) * lda];
      }
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (base + 256 * q < total) buf[base + 256 * q] = v[q];
  }
  __syncthreads();
  for (int idx = tid; idx < total; idx += 256) {
    const int m = idx % nm, c = idx / nm;
    A[smv[2 * m] + (long)(c0 + c) * lda] = buf[idx];
  }
}

// dense copy of op-free triangle: D = tri(A) with unit/zero handling
__global__ void tri_to_dense_kernel(int n, const double *A, long lda, double *D, int uplo, int unit) {
  long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % n), j = (int)(idx / n);
    double v;
    if (i == j) v = unit ? 1.0 : A[i + (long)j * lda];
    else if ((uplo == kLower) == (i > j)) v = A[i + (long)j * lda];
    else v = 0.0;
    D[idx] = v;
  }
}

template <typename T>
__global__ void copy2d_kernel(int M, int N, const T *S, long lds, T *D, long ldd) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    D[i + (long)j * ldd] = S[i + (long)j * lds];
  }
}

template <typename T>
__global__ void fill_zero_kernel(T *A, int M, int N, long lda) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x)
    A[(idx % M) + (idx / M) * lda] = T(0);
}

__global__ void set_info_kernel(int *d) { *d = 0x7fffffff; }
__global__ void finish_info_kernel(int *d) { if (*d == 0x7fffffff) *d = 0; }

}  // namespace

template <typename T>
void trinv_dev(int n, const T *Tp, long tr, long tc, int lower, int unit, T *W, cudaStream_t st) {
  constexpr int smem = 3 * LEAF * (LEAF + 1) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trinv_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  trinv_kernel<T><<<cdiv(n, LEAF), 256, smem, st>>>(n, Tp, tr, tc, lower, unit, W);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trinv_dev<double>(int, const double *, long, long, int, int, double *, cudaStream_t);
template void trinv_dev<float>(int, const float *, long, long, int, int, float *, cudaStream_t);

// The solve proper; W receives the inverted diagonal blocks (ceil(n/64)
// blocks of 64x64 elements, n = order of the triangle).
template <typename T>
void trsm_impl(int side, int uplo, int trans, int diag, int M, int N, T alpha, const T *A, long lda,
               T *B, long ldb, cudaStream_t st, SgemmFn gemm, T *W) {
  if (M <= 0 || N <= 0) return;
  const bool tr = trans != kNoTrans;
  Eff<T> e;
  e.Tp = A;
  e.unit = diag == kUnit;
  int n, m;
  const bool opLower = (uplo == kLower) != tr;  // op(A) lower triangular?
  if (side == kLeft) {  // op(A) X = B
    e.tr = tr ? lda : 1; e.tc = tr ? 1 : lda;
    e.Bp = B; e.br = 1; e.bc = ldb;
    e.lower = opLower;
    n = M; m = N;
  } else {  // X op(A) = B  <=>  op(A)^T X^T = B^T
    e.tr = tr ? 1 : lda; e.tc = tr ? lda : 1;
    e.Bp = B; e.br = ldb; e.bc = 1;
    e.lower = !opLower;
    n = N; m = M;
  }
  if (alpha == T(0)) { fill_zero_dev<T>(B, M, N, ldb, st); return; }
  if (alpha != T(1)) {
    long total = (long)n * m;
    scale_strided_kernel<T><<<(int)std::min<long>((total + 255) / 256, 4096), 256, 0, st>>>(
        n, m, alpha, e.Bp, e.br, e.bc);
    ATLB_CUDA_CHECK(cudaGetLastError());
  }
  const int nblk = cdiv(n, LEAF);
  (void)nblk;
  trinv_dev<T>(n, e.Tp, e.tr, e.tc, e.lower, e.unit, W, st);
  e.W = W;
  eff_solve(e, 0, n, m, gemm, st);
}

template void trsm_impl<double>(int, int, int, int, int, int, double, const double *, long, double *,
                                long, cudaStream_t, SgemmFn, double *);

template <typename T>
void trsm_dev(int side, int uplo, int trans, int diag, int M, int N, T alpha, const T *A, long lda,
              T *B, long ldb, cudaStream_t st, SgemmFn gemm) {
  if (M <= 0 || N <= 0) return;
  const int n = side == kLeft ? M : N;
  T *W = (T *)scratch(kSlotTrsmW, sizeof(T) * (size_t)cdiv(n, LEAF) * LEAF * LEAF);
  trsm_impl<T>(side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb, st, gemm, W);
}

template void trsm_dev<double>(int, int, int, int, int, int, double, const double *, long,
                               double *, long, cudaStream_t, SgemmFn);
template void trsm_dev<float>(int, int, int, int, int, int, float, const float *, long, float *,
                              long, cudaStream_t, SgemmFn);

namespace {
// X = L^-1 B in place, L unit lower triangular of order m <= 256, B m x n:
// the U12 = L11^-1 A12 step of the blocked LU in ONE launch (the recursive
// trsm_dev issues a TRSM/GEMM cascade of ~8 kernels for it).  CTA q solves
// columns 32q .. 32q+31, the whole column tile in shared memory: for each
// 32-row block, the product of L's 32 x (32 ib) panel with the rows already
// solved (L read in 32 x 32 tiles, the next tile fetched into registers while
// the current one is used), then forward substitution with the unit lower
// 32 x 32 diagonal tile (lane = row, x_k by shuffle, four columns per warp).
constexpr int LLU_COLS = 32, LLU_MAX = 256;

template <typename T>
__global__ void __launch_bounds__(256, 1)
trsm_llu_small_kernel(int m, int n, const T *__restrict__ L, long lda, T *B, long ldb) {
  extern __shared__ __align__(16) unsigned char llu_smem[];
  T(*sX)[LLU_COLS + 1] = reinterpret_cast<T(*)[LLU_COLS + 1]>(llu_smem);  // [LLU_MAX]: B, then X
  T(*sL)[33] = reinterpret_cast<T(*)[33]>(sX + LLU_MAX);                  // [32]: one tile of L
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.x * LLU_COLS, nc = min(LLU_COLS, n - c0);
  for (int base = 0; base < LLU_MAX * LLU_COLS; base += 256 * 8) {  // eight loads in flight per thread
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, r = idx % LLU_MAX, c = idx / LLU_MAX;
      v[u] = (r < m && c < nc) ? B[r + (long)(c0 + c) * ldb] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid;
      sX[idx % LLU_MAX][idx / LLU_MAX] = v[u];
    }
  }
  const int nblk = (m + 31) / 32;
  const int rr = tid % 32, cq = tid / 32;  // update: row rr of the block, columns 4 cq .. 4 cq + 3
  // a thread's four elements of an L tile (rows r0 + i, columns k0 + k)
  auto fetch = [&](int r0, int k0, T (&v)[4]) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int idx = tid + 256 * e, i = idx % 32, k = idx / 32;
      v[e] = (r0 + i < m && k0 + k < m) ? L[r0 + i + (long)(k0 + k) * lda] : T(0);
    }
  };
  auto store = [&](const T (&v)[4]) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int idx = tid + 256 * e;
      sL[idx % 32][idx / 32] = v[e];
    }
  };
  for (int ib = 0; ib < nblk; ib++) {
    const int r0 = ib * 32;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    T nxt[4];
    fetch(r0, 0, nxt);  // tile (ib, 0), or the diagonal tile when ib == 0
    for (int kt = 0; kt < ib; kt++) {
      __syncthreads();  // the previous tile has been used
      store(nxt);
      __syncthreads();
      fetch(r0, (kt + 1) * 32, nxt);  // the next tile (the diagonal one after the last)
#pragma unroll 8
      for (int k = 0; k < 32; k++) {
        const T lv = sL[rr][k];
#pragma unroll
        for (int e = 0; e < 4; e++) acc[e] = fma(lv, sX[kt * 32 + k][4 * cq + e], acc[e]);
      }
    }
    __syncthreads();  // every thread is done with sL and the rows it read
#pragma unroll
    for (int e = 0; e < 4; e++) sX[r0 + rr][4 * cq + e] -= acc[e];
    store(nxt);       // the diagonal tile
    __syncthreads();
    T x[4];
#pragma unroll
    for (int e = 0; e < 4; e++) x[e] = sX[r0 + lane][4 * warp + e];
#pragma unroll
    for (int k = 0; k < 31; k++) {
      const T lk = sL[lane][k];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const T xk = __shfl_sync(0xffffffffu, x[e], k);
        if (lane > k) x[e] = fma(-lk, xk, x[e]);
      }
    }
#pragma unroll
    for (int e = 0; e < 4; e++) sX[r0 + lane][4 * warp + e] = x[e];
    __syncthreads();
  }
  for (int idx = tid; idx < LLU_MAX * LLU_COLS; idx += 256) {
    const int r = idx % LLU_MAX, c = idx / LLU_MAX;
    if (r < m && c < nc) B[r + (long)(c0 + c) * ldb] = sX[r][c];
  }
}

// The same solve in FP32 (the factorization inside the mixed solvers), with
// no global load on its dependency chain: L's lower 32 x 32 tiles (at most 36,
// 144 KB) reach shared memory in one burst of cp.async copies, warp w inverts
// the unit lower diagonal tile w (lane i solves row i of the inverse,
// y L = e_i, by backward substitution), and block row ib is then
//   X_ib = inv(L_ib,ib) (B_ib - sum_{kt < ib} L_ib,kt X_kt),
// 32-term dot products instead of the 31-step shuffle chain.  Entries of L
// above the diagonal (U's, in a packed LU) are never read.  NCOL = 8 CPT
// columns per CTA, CPT per thread: 256 columns spread over 32 CTAs.  With
// KS = 2 (the narrow look-ahead block, one column per thread) each 32-term
// product is split between two warps, whose halves meet in shared memory:
// twice the warps per CTA to hide the chain's latency.
// Tile (ib, kt) sits at t = ib (ib + 1) / 2 + kt, stored [k][i] = L[32 ib + i][32 kt + k]
// (lane = row: conflict-free reads).
constexpr int LLI_TILES = 36;

template <int CPT, int KS>
__global__ void __launch_bounds__(256 * KS, 1)
trsm_llu_inv_kernel(int m, int n, const float *__restrict__ L, long lda, float *B, long ldb) {
  constexpr int NCOL = 8 * CPT;
  extern __shared__ __align__(16) unsigned char lli_smem[];
  float *sLT = reinterpret_cast<float *>(lli_smem);  // the tiles, 1024 floats each
  float *sX = sLT + LLI_TILES * 1024;                 // [NCOL][256]: B, then X
  float *sY = sX + NCOL * LLU_MAX;                    // [NCOL][32]: one block row before inv(L_ib,ib)
  float *sP = sY + NCOL * 32;                         // [KS][NCOL][32]: the k-range halves' sums (KS = 2)
  constexpr int NT = 256 * KS, KR = 32 / KS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cw = warp & 7, h = warp >> 3, kb = h * KR;  // columns cw + 8 e, k in [kb, kb + KR) of each tile
  const int c0 = blockIdx.x * NCOL, nc = min(NCOL, n - c0);
  const int nblk = (m + 31) / 32;
  for (int ib = 0; ib < nblk; ib++)
    for (int kt = 0; kt <= ib; kt++) {
      float *dst = sLT + (ib * (ib + 1) / 2 + kt) * 1024;
      for (int e = tid; e < 1024; e += NT) {
        const int k = e >> 5, i = e & 31, r = 32 * ib + i, c = 32 * kt + k;
        const bool ok = r < m && c < m && (kt < ib || i > k);  // strictly lower, zero elsewhere
        cp_async4(dst + e, ok ? L + r + (long)c * lda : L, ok);
      }
    }
  for (int e = tid; e < NCOL * LLU_MAX; e += NT) {
    const int c = e / LLU_MAX, r = e % LLU_MAX;
    const bool ok = r < m && c < nc;
    cp_async4(sX + e, ok ? B + r + (long)(c0 + c) * ldb : B, ok);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if (warp < nblk) {
    float *D = sLT + (warp * (warp + 1) / 2 + warp) * 1024;
    float y[32];
#pragma unroll
    for (int k = 31; k >= 0; k--) {
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int j = k + 1; j < 32; j++) {
        if ((j - k) & 1) s0 = fmaf(y[j], D[k * 32 + j], s0);
        else s1 = fmaf(y[j], D[k * 32 + j], s1);
      }
      y[k] = k == lane ? 1.f : (k > lane ? 0.f : -(s0 + s1));
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 32; k++) D[k * 32 + lane] = y[k];  // inv(L)[lane][k], same layout
  }
  __syncthreads();
  for (int ib = 0; ib < nblk; ib++) {
    const int r0 = 32 * ib;
    float acc[CPT][2];
#pragma unroll
    for (int e = 0; e < CPT; e++) acc[e][0] = acc[e][1] = 0.f;
    for (int kt = 0; kt < ib; kt++) {
      const float *T = sLT + (ib * (ib + 1) / 2 + kt) * 1024;
#pragma unroll 4
      for (int k = kb; k < kb + KR; k += 4) {
        float lv[4];
#pragma unroll
        for (int q = 0; q < 4; q++) lv[q] = T[(k + q) * 32 + lane];
#pragma unroll
        for (int e = 0; e < CPT; e++) {
          const float4 xv = *reinterpret_cast<const float4 *>(sX + (cw + 8 * e) * LLU_MAX + 32 * kt + k);
          acc[e][0] = fmaf(lv[0], xv.x, acc[e][0]);
          acc[e][1] = fmaf(lv[1], xv.y, acc[e][1]);
          acc[e][0] = fmaf(lv[2], xv.z, acc[e][0]);
          acc[e][1] = fmaf(lv[3], xv.w, acc[e][1]);
        }
      }
    }
    if constexpr (KS == 1) {
#pragma unroll
      for (int e = 0; e < CPT; e++) {
        const int c = cw + 8 * e;
        sY[c * 32 + lane] = sX[c * LLU_MAX + r0 + lane] - (acc[e][0] + acc[e][1]);
      }
    } else {
#pragma unroll
      for (int e = 0; e < CPT; e++) sP[(h * NCOL + cw + 8 * e) * 32 + lane] = acc[e][0] + acc[e][1];
      __syncthreads();
      if (h == 0) {
#pragma unroll
        for (int e = 0; e < CPT; e++) {
          const int c = cw + 8 * e;
          sY[c * 32 + lane] = sX[c * LLU_MAX + r0 + lane] - (sP[c * 32 + lane] + sP[(NCOL + c) * 32 + lane]);
        }
      }
    }
    __syncthreads();
    const float *D = sLT + (ib * (ib + 1) / 2 + ib) * 1024;
#pragma unroll
    for (int e = 0; e < CPT; e++) acc[e][0] = acc[e][1] = 0.f;
#pragma unroll 4
    for (int k = kb; k < kb + KR; k += 4) {
      float lv[4];
#pragma unroll
      for (int q = 0; q < 4; q++) lv[q] = D[(k + q) * 32 + lane];
#pragma unroll
      for (int e = 0; e < CPT; e++) {
        const float4 yv = *reinterpret_cast<const float4 *>(sY + (cw + 8 * e) * 32 + k);
        acc[e][0] = fmaf(lv[0], yv.x, acc[e][0]);
        acc[e][1] = fmaf(lv[1], yv.y, acc[e][1]);
        acc[e][0] = fmaf(lv[2], yv.z, acc[e][0]);
        acc[e][1] = fmaf(lv[3], yv.w, acc[e][1]);
      }
    }
    if constexpr (KS == 1) {
#pragma unroll
      for (int e = 0; e < CPT; e++) sX[(cw + 8 * e) * LLU_MAX + r0 + lane] = acc[e][0] + acc[e][1];
    } else {
#pragma unroll
      for (int e = 0; e < CPT; e++) sP[(h * NCOL + cw + 8 * e) * 32 + lane] = acc[e][0] + acc[e][1];
      __syncthreads();
      if (h == 0) {
#pragma unroll
        for (int e = 0; e < CPT; e++) {
          const int c = cw + 8 * e;
          sX[c * LLU_MAX + r0 + lane] = sP[c * 32 + lane] + sP[(NCOL + c) * 32 + lane];
        }
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < NCOL * LLU_MAX; e += NT) {
    const int c = e / LLU_MAX, r = e % LLU_MAX;
    if (r < m && c < nc) B[r + (long)(c0 + c) * ldb] = sX[e];
  }
}

template <int CPT, int KS>
void trsm_llu_inv_launch(int m, int n, const float *L, long lda, float *B, long ldb, cudaStream_t st) {
  constexpr int smem = (LLI_TILES * 1024 + 8 * CPT * (LLU_MAX + 32 + 32 * KS)) * (int)sizeof(float);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsm_llu_inv_kernel<CPT, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem));
    configured = true;
  }
  trsm_llu_inv_kernel<CPT, KS><<<cdiv(n, 8 * CPT), 256 * KS, smem, st>>>(m, n, L, lda, B, ldb);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
}  // namespace

template <typename T>
void trsm_llu_small_dev(int m, int n, const T *L, long lda, T *B, long ldb, cudaStream_t st) {
  if (m <= 0 || n <= 0) return;
  if (sizeof(T) == 4) {  // FP32: L in shared memory, inverted diagonal tiles
    if (n <= 8 * num_sms()) trsm_llu_inv_launch<1, 2>(m, n, (const float *)L, lda, (float *)B, ldb, st);
    else trsm_llu_inv_launch<4, 1>(m, n, (const float *)L, lda, (float *)B, ldb, st);
    return;
  }
  constexpr int smem = (LLU_MAX * (LLU_COLS + 1) + 32 * 33) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsm_llu_small_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  trsm_llu_small_kernel<T><<<cdiv(n, LLU_COLS), 256, smem, st>>>(m, n, L, lda, B, ldb);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trsm_llu_small_dev<double>(int, int, const double *, long, double *, long, cudaStream_t);
template void trsm_llu_small_dev<float>(int, int, const float *, long, float *, long, cudaStream_t);

void dtrmm_dev(int side, int uplo, int trans, int diag, int M, int N, double alpha,
               const double *A, long lda, double *B, long ldb, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  int n = side == kLeft ? M : N;
  double *D = (double *)scratch(kSlotWork2, sizeof(double) * ((size_t)n * n + (size_t)M * N));
  double *W = D + (size_t)n * n;
  long tot = (long)n * n;
  tri_to_dense_kernel<<<(int)std::min<long>((tot + 255) / 256, 4096), 256, 0, st>>>(
      n, A, lda, D, uplo, diag == kUnit);
  ATLB_CUDA_CHECK(cudaGetLastError());
  if (side == kLeft)
    dgemm_dev(trans, kNoTrans, M, N, M, alpha, D, n, B, ldb, 0.0, W, M, st);
  else
    dgemm_dev(kNoTrans, trans, M, N, N, alpha, B, ldb, D, n, 0.0, W, M, st);
  long tot2 = (long)M * N;
  copy2d_kernel<double><<<(int)std::min<long>((tot2 + 255) / 256, 4096), 256, 0, st>>>(M, N, W, M, B, ldb);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void laswp_dev(int ncols, T *A, long lda, int k1, int k2, const int *ipiv, int inc,
               cudaStream_t st) {
  if (ncols <= 0 || k2 <= k1) return;
  int *ws = (int *)scratch(kSlotLaswp, sizeof(int) * (4 * LSW_MAXP + 64));
  int *moves = ws + 64, *nmoves = ws, *ok = ws + 1;
  constexpr int smem = 2 * LSW_MAXP * LSW_COLS * (int)sizeof(T) + 4 * LSW_MAXP * (int)sizeof(int);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(laswp_apply_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(laswp_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         LSW_SPAN * (int)sizeof(int)));
    configured = true;
  }
  // columns per CTA: enough CTAs to cover the GPU twice, at most LSW_COLS
  const int cpc = std::max(1, std::min(LSW_COLS, ncols / (2 * num_sms())));
  const int nchunk = cdiv(k2 - k1, LSW_MAXP);
  for (int ci = 0; ci < nchunk; ci++) {
    const int ch = inc > 0 ? ci : nchunk - 1 - ci;
    const int a = k1 + ch * LSW_MAXP, b = std::min(k2, a + LSW_MAXP);
    laswp_plan_kernel<<<1, 1024, LSW_SPAN * sizeof(int), st>>>(a, b, ipiv, inc, moves, nmoves, ok);
    laswp_apply_kernel<T><<<cdiv(ncols, cpc), 256, smem, st>>>(ncols, cpc, A, lda, moves, nmoves, ok, a, b,
                                                               ipiv, inc);
  }
  ATLB_CUDA_CHECK(cudaGetLastError());
}

namespace {
// The net row permutation of n interchanges (perm[i] = the original row that
// ends at position i), in two launches instead of one n-step chain:
//  1. perm_plan_kernel, one CTA per chunk of 256 interchanges, all chunks at
//     once: a chunk touches its own 256 positions and the distinct pivot rows
//     below them (at most 256 more), so its net effect is a permutation of at
//     most 512 slots; thread 0 replays the chunk's swaps on the slots and
//     slot s leaves as the pair (destination, source) (destination -1 for an
//     unused slot);
//  2. perm_compose_kernel, one CTA: the chunks' pairs applied in order to the
//     index vector (all sources read, barrier, all destinations written).
constexpr int PP_CHUNK = 256;

__global__ void __launch_bounds__(PP_CHUNK)
perm_plan_kernel(int n, const int *__restrict__ ipiv, int *__restrict__ moves) {
  __shared__ int sp[PP_CHUNK], bslot[PP_CHUNK];
  __shared__ int pos[2 * PP_CHUNK], val[2 * PP_CHUNK];
  const int tid = threadIdx.x, k1 = blockIdx.x * PP_CHUNK, nk = min(PP_CHUNK, n - k1), k2 = k1 + nk;
  if (tid < nk) sp[tid] = ipiv[k1 + tid];
  pos[tid] = tid < nk ? k1 + tid : -1;
  pos[PP_CHUNK + tid] = -1;
  __syncthreads();
  if (tid < nk) {
    const int p = sp[tid];
    int s = tid;                           // an interchange outside [k1, n) is skipped
    if (p >= k1 && p < k2) s = p - k1;
    else if (p >= k2 && p < n) {
      int first = tid;                     // the slot of a pivot row is its first occurrence's
      for (int q = 0; q < tid; q++)
        if (sp[q] == p) { first = q; break; }
      s = PP_CHUNK + first;
      if (first == tid) pos[s] = p;
    }
    bslot[tid] = s;
  }
  __syncthreads();
  val[tid] = pos[tid];
  val[PP_CHUNK + tid] = pos[PP_CHUNK + tid];
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < nk; k++) {
      const int b = bslot[k], t = val[k];
      val[k] = val[b];
      val[b] = t;
    }
  __syncthreads();
  int *mv = moves + (long)blockIdx.x * 4 * PP_CHUNK;
  for (int s = tid; s < 2 * PP_CHUNK; s += PP_CHUNK) {
    mv[2 * s] = pos[s];
    mv[2 * s + 1] = val[s];
  }
}

__global__ void __launch_bounds__(1024)
perm_compose_kernel(int n, int nchunk, const int *__restrict__ moves, int *__restrict__ perm, int use_smem) {
  extern __shared__ int spv[];
  int *pv = use_smem ? spv : perm;
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) pv[i] = i;
  int d = -1, s = 0;
  if (tid < 2 * PP_CHUNK) { d = moves[2 * tid]; s = moves[2 * tid + 1]; }
  __syncthreads();
  for (int c = 0; c < nchunk; c++) {
    int dn = -1, sn = 0;  // the next chunk's pair, fetched while this one is applied
    if (tid < 2 * PP_CHUNK && c + 1 < nchunk) {
      const int *mv = moves + (long)(c + 1) * 4 * PP_CHUNK;
      dn = mv[2 * tid];
      sn = mv[2 * tid + 1];
    }
    const int v = d >= 0 ? pv[s] : 0;
    __syncthreads();
    if (d >= 0) pv[d] = v;
    __syncthreads();
    d = dn;
    s = sn;
  }
  if (use_smem)
    for (int i = tid; i < n; i += blockDim.x) perm[i] = pv[i];
}
}  // namespace

void ipiv_to_perm_dev(int n, const int *ipiv, int *perm, cudaStream_t st) {
  if (n <= 0) return;
  const int nchunk = cdiv(n, PP_CHUNK);
  int *moves = (int *)scratch(kSlotPermPlan, sizeof(int) * 4 * PP_CHUNK * (size_t)nchunk);
  const size_t bytes = sizeof(int) * (size_t)n;
  const int use_smem = bytes <= 200 * 1024;
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(perm_compose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    configured = true;
  }
  perm_plan_kernel<<<nchunk, PP_CHUNK, 0, st>>>(n, ipiv, moves);
  perm_compose_kernel<<<1, 1024, use_smem ? bytes : 0, st>>>(n, nchunk, moves, perm, use_smem);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

template void laswp_dev<double>(int, double *, long, int, int, const int *, int, cudaStream_t);
template void laswp_dev<float>(int, float *, long, int, int, const int *, int, cudaStream_t);

template <typename T>
void fill_zero_dev(T *A, int M, int N, long lda, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  long total = (long)M * N;
  fill_zero_kernel<T><<<(int)std::min<long>((total + 255) / 256, 4096), 256, 0, st>>>(A, M, N, lda);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void fill_zero_dev<double>(double *, int, int, long, cudaStream_t);
template void fill_zero_dev<float>(float *, int, int, long, cudaStream_t);

void set_info_kernel_launch(int *d, cudaStream_t st) { set_info_kernel<<<1, 1, 0, st>>>(d); }
void finish_info_kernel_launch(int *d, cudaStream_t st) { finish_info_kernel<<<1, 1, 0, st>>>(d); }

}  // namespace atlb
