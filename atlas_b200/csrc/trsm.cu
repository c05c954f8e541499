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

// B2 (n2 x m) -= T21 (n2 x n1) * X1 (n1 x m), everything in effective strides.
template <typename T>
void eff_update(const Eff<T> &e, int r2, int n2, int r1, int n1, int m, SgemmFn fn,
                cudaStream_t st) {
  const T *T21 = e.Tp + r2 * e.tr + r1 * e.tc;
  T *B2 = e.Bp + r2 * e.br;
  const T *X1 = e.Bp + r1 * e.br;
  if (e.br == 1) {  // B column-major (ld = bc)
    int ta = (e.tr == 1) ? kNoTrans : kTrans;
    long ldt = (e.tr == 1) ? e.tc : e.tr;
    gemm_call<T>(fn, ta, kNoTrans, n2, m, n1, T(-1), T21, ldt, X1, e.bc, T(1), B2, e.bc, st);
  } else {  // B^T column-major (m x n) with ld = br: B2^T -= X1^T * T21^T
    int tb = (e.tc == 1) ? kNoTrans : kTrans;
    long ldt = (e.tc == 1) ? e.tr : e.tc;
    gemm_call<T>(fn, kNoTrans, tb, m, n2, n1, T(-1), X1, e.br, T21, ldt, T(1), B2, e.br, st);
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
// kernel then moves only those rows, in parallel over columns (16 per CTA):
// all sources are read into shared memory before any destination is written,
// so the in-place permutation needs no ordering.
constexpr int LSW_MAXP = 256;               // pivots per plan
constexpr int LSW_SPAN = 24576;             // rows a plan can track in shared memory
constexpr int LSW_COLS = 16;

__global__ void __launch_bounds__(1024)
laswp_plan_kernel(int k1, int k2, const int *__restrict__ ipiv, int inc, int *__restrict__ moves,
                  int *__restrict__ nmoves, int *__restrict__ ok) {
  extern __shared__ int perm[];  // LSW_SPAN entries
  __shared__ int s_hi, s_cnt;
  const int tid = threadIdx.x;
  if (tid == 0) { s_hi = k2; s_cnt = 0; }
  __syncthreads();
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

template <typename T>
__global__ void __launch_bounds__(256)
laswp_apply_kernel(int ncols, T *A, long lda, const int *__restrict__ moves, const int *__restrict__ nmoves) {
  extern __shared__ __align__(16) unsigned char lsw_smem[];
  T *buf = reinterpret_cast<T *>(lsw_smem);  // [2*LSW_MAXP][LSW_COLS]
  const int nm = *nmoves, c0 = blockIdx.x * LSW_COLS, tid = threadIdx.x;
  const int nc = min(LSW_COLS, ncols - c0);
  // moves fastest: neighbouring threads take neighbouring (sorted) rows of one column
  for (int idx = tid; idx < nm * LSW_COLS; idx += 256) {
    const int m = idx % nm, c = idx / nm;
    if (c < nc) buf[idx] = A[moves[2 * m + 1] + (long)(c0 + c) * lda];
  }
  __syncthreads();
  for (int idx = tid; idx < nm * LSW_COLS; idx += 256) {
    const int m = idx % nm, c = idx / nm;
    if (c < nc) A[moves[2 * m] + (long)(c0 + c) * lda] = buf[idx];
  }
}

// Sequential fallback (one thread per column) for pivots spread over more
// rows than a plan can track.
template <typename T>
__global__ void __launch_bounds__(256)
laswp_seq_kernel(int ncols, T *A, long lda, int k1, int k2, const int *__restrict__ ipiv, int inc,
                 const int *__restrict__ ok) {
  if (*ok) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  T *col = A + (long)c * lda;
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
  for (int idx = tid; idx < LLU_MAX * LLU_COLS; idx += 256) {
    const int r = idx % LLU_MAX, c = idx / LLU_MAX;
    sX[r][c] = (r < m && c < nc) ? B[r + (long)(c0 + c) * ldb] : T(0);
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
}  // namespace

template <typename T>
void trsm_llu_small_dev(int m, int n, const T *L, long lda, T *B, long ldb, cudaStream_t st) {
  if (m <= 0 || n <= 0) return;
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
  constexpr int smem = 2 * LSW_MAXP * LSW_COLS * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(laswp_apply_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(laswp_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         LSW_SPAN * (int)sizeof(int)));
    configured = true;
  }
  const int nchunk = cdiv(k2 - k1, LSW_MAXP);
  for (int ci = 0; ci < nchunk; ci++) {
    const int ch = inc > 0 ? ci : nchunk - 1 - ci;
    const int a = k1 + ch * LSW_MAXP, b = std::min(k2, a + LSW_MAXP);
    laswp_plan_kernel<<<1, 1024, LSW_SPAN * sizeof(int), st>>>(a, b, ipiv, inc, moves, nmoves, ok);
    laswp_apply_kernel<T><<<cdiv(ncols, LSW_COLS), 256, smem, st>>>(ncols, A, lda, moves, nmoves);
    laswp_seq_kernel<T><<<cdiv(ncols, 256), 256, 0, st>>>(ncols, A, lda, a, b, ipiv, inc, ok);
  }
  ATLB_CUDA_CHECK(cudaGetLastError());
}

namespace {
// One thread replays the n interchanges on an index vector (the chain is
// sequential); the vector sits in shared memory when it fits.
__global__ void ipiv_perm_kernel(int n, const int *__restrict__ ipiv, int *__restrict__ perm, int use_smem) {
  extern __shared__ int sp[];
  int *pv = use_smem ? sp : perm;
  int *ip = use_smem ? sp + n : nullptr;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    pv[i] = i;
    if (use_smem) ip[i] = ipiv[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < n; k++) {
      const int b = use_smem ? ip[k] : ipiv[k];
      const int t = pv[k];
      pv[k] = pv[b];
      pv[b] = t;
    }
  }
  __syncthreads();
  if (use_smem)
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = pv[i];
}
}  // namespace

void ipiv_to_perm_dev(int n, const int *ipiv, int *perm, cudaStream_t st) {
  if (n <= 0) return;
  const size_t bytes = sizeof(int) * 2 * (size_t)n;
  const int use_smem = bytes <= 200 * 1024;
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(ipiv_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    configured = true;
  }
  ipiv_perm_kernel<<<1, 1024, use_smem ? bytes : 0, st>>>(n, ipiv, perm, use_smem);
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
