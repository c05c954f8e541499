// Triangular solve for a few right-hand sides (NRHS <= 8) in ONE launch.
//
// The recursive TRSM (trsm.cu) issues ~2n/64 launches, which for one
// right-hand side is all latency.  Here one CTA owns one 128-row block of
// the solution (two 64-row sub-blocks): it takes a ticket from an atomic
// counter (tickets are handed out in launch order, so every block it depends
// on is owned by a CTA that is already running and never waits on it) and
// accumulates the products with the solved blocks.  The blocks solved long
// ago are streamed in bulk: one warp looks up to 32 "done" flags at once
// and the CTA then runs through every block found done without waiting
// again; only the block just before it is awaited, with its matrix values
// already in registers.  The block is then solved by one product with the
// inverse of its 128 x 128 diagonal block (computed once per factor by
// trsv_inverse_dev, loaded into shared memory before any wait) and
// published.  In FP32 the block just before is not awaited through its flag:
// its x also goes out as (value, epoch) 64-bit words, each written by one
// single-copy-atomic store, and the next block polls those words directly --
// one round trip to L2 on the chain instead of fence, flag and data load.
// Every wait is bounded: after ~1 s the kernel records an error in *err and
// stops waiting (the result is then wrong but the GPU is released).  The
// launcher clears the ticket counter, the flags and the tagged words before
// each launch.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int BS = 64;       // rows of a diagonal block (W's blocks)
constexpr int CB = 2 * BS;   // rows of one CTA's block
constexpr int TT = 512;      // threads: four per row of the CTA's block
constexpr int NQ = TT / CB;  // parts a row's dot products are split into
constexpr int PART = CB / NQ;  // columns of a solved block per thread

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T, int NR>
__global__ void __launch_bounds__(TT, 1)
trsv_kernel(int n, int nrhs, const T *__restrict__ Tp, long tr, long tc, int lower,
            const T *__restrict__ W, T *X, long ldx, int *counter, int *flags, int epoch, int *err,
            unsigned long long *xt) {
  extern __shared__ __align__(16) unsigned char trsv_smem[];
  T(*sW)[CB + 1] = reinterpret_cast<T(*)[CB + 1]>(trsv_smem);   // [CB]: the inverted diagonal block
  T(*sxd)[CB][NR] = reinterpret_cast<T(*)[CB][NR]>(sW + CB);    // x of a solved block, double-buffered
  T(*sb)[NR] = reinterpret_cast<T(*)[NR]>(sxd + 2);             // this block's b
  T(*sacc)[CB][NR] = reinterpret_cast<T(*)[CB][NR]>(sb + CB);   // [NQ]: the parts' sums
  __shared__ int s_bi, s_ready;
  const int tid = threadIdx.x, lane = tid & 31, nb = (n + CB - 1) / CB;
  if (tid == 0) {
    const int t = atomicAdd(counter, 1);
    s_bi = lower ? t : nb - 1 - t;
  }
  __syncthreads();
  const int bi = s_bi, r0 = bi * CB, rows = min(CB, n - r0);
  // everything that does not depend on other blocks is fetched first
  {
    const T *Wb = W + (long)bi * CB * CB;  // column-major 128 x 128
    for (int base = tid; base < CB * CB; base += 8 * TT) {  // eight loads in flight per thread
      T v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = Wb[base + q * TT];
#pragma unroll
      for (int q = 0; q < 8; q++) sW[(base + q * TT) % CB][(base + q * TT) / CB] = v[q];
    }
  }
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    sb[rr][q] = (rr < rows && q < nrhs) ? X[r0 + rr + (long)q * ldx] : T(0);
  }
  // thread (row, part): row of this block, columns part*PART .. +PART-1 of every solved block
  const int row = tid % CB, part = tid / CB;
  const T *trow = Tp + (long)(r0 + row) * tr;
  const int ndep = lower ? bi : nb - 1 - bi;
  T acc[NR], acc2[NR];  // even and odd columns: two independent FMA chains
#pragma unroll
  for (int q = 0; q < NR; q++) acc[q] = acc2[q] = T(0);
  auto wait_flag = [&](int bj) {
    const uint64_t t0 = gtimer();
    while (ld_acquire(flags + bj) != epoch) {
      if (gtimer() - t0 > 1000000000ull) { atomicExch(err, 1); break; }
    }
  };
  // x of block bj into sxd[buf] (all threads), then the products
  auto load_x = [&](int bj, int buf) {
    const int c0 = bj * CB;
    for (int idx = tid; idx < CB * NR; idx += TT) {
      const int cc = idx % CB, q = idx / CB;
      sxd[buf][cc][q] = (c0 + cc < n && q < nrhs) ? __ldcg(X + c0 + cc + (long)q * ldx) : T(0);
    }
  };
  // 1. solved blocks in bulk: all but the last dependency
  int d = 0, buf = 0;
  while (d < ndep - 1) {
    if (tid < 32) {
      // how many of the next blocks (up to 32, never the last one) are done
      const int dd = d + lane;
      const bool ok = dd < ndep - 1 && ld_acquire(flags + (lower ? dd : nb - 1 - dd)) == epoch;
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      const int ready = __ffs(~m) - 1;  // leading run of done blocks
      if (lane == 0) {
        if (ready == 0) wait_flag(lower ? d : nb - 1 - d);
        s_ready = ready == 0 ? 1 : ready;
      }
    }
    __syncthreads();
    const int nr = s_ready;
    for (int e = 0; e < nr; e++, d++) {
      const int bj = lower ? d : nb - 1 - d;
      const int c0 = bj * CB + part * PART, cols = min(PART, n - c0);
      // all of this thread's matrix loads in flight at once, issued before
      // the barrier: a CTA far down the triangle streams many blocks, and
      // this stream (not the chain of solves) bounds it when fewer loads
      // are in flight
      T tv[PART];
#pragma unroll
      for (int k = 0; k < PART; k++) tv[k] = (row < rows && k < cols) ? trow[(long)(c0 + k) * tc] : T(0);
      load_x(bj, buf);
      __syncthreads();
      const T(*xs)[NR] = sxd[buf] + part * PART;
#pragma unroll
      for (int k = 0; k < PART; k += 2)
#pragma unroll
        for (int q = 0; q < NR; q++) {
          acc[q] = fma(tv[k], xs[k][q], acc[q]);
          acc2[q] = fma(tv[k + 1], xs[k + 1][q], acc2[q]);
        }
      buf ^= 1;
    }
    __syncthreads();  // s_ready is read by every thread before it is rewritten
  }
  // 2. the block just before this one: its matrix values first, then the wait
  if (ndep > 0) {
    const int bj = lower ? ndep - 1 : nb - ndep;
    const int c0 = bj * CB + part * PART, cols = min(PART, n - c0);
    T tv[PART];
#pragma unroll
    for (int k = 0; k < PART; k++) tv[k] = (row < rows && k < cols) ? trow[(long)(c0 + k) * tc] : T(0);
    if constexpr (sizeof(T) == 4) {
      // FP32: x arrives as (value, epoch) 64-bit words, each written by one
      // single-copy-atomic store, so a word whose tag is current carries its
      // value: one round trip to L2 instead of flag, fence and data
      const uint64_t t0 = gtimer();
      while (true) {
        bool ok = true;
        for (int idx = tid; idx < CB * NR; idx += TT) {
          const int cc = idx % CB, q = idx / CB;
          T v = T(0);
          if (bj * CB + cc < n && q < nrhs) {
            const unsigned long long w = __ldcg(xt + (long)(bj * CB + cc) * NR + q);
            ok = ok && (int)(w >> 32) == epoch;
            v = __uint_as_float((unsigned)(w & 0xffffffffu));
          }
          sxd[buf][cc][q] = v;
        }
        if (__syncthreads_and(ok)) break;
        if (gtimer() - t0 > 1000000000ull) {  // bounded: record and go on (the result is then wrong)
          if (tid == 0) atomicExch(err, 1);
          break;
        }
      }
    } else {
      if (tid == 0) wait_flag(bj);
      __syncthreads();
      load_x(bj, buf);
      __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < PART; k += 2)
#pragma unroll
      for (int q = 0; q < NR; q++) {
        acc[q] = fma(tv[k], sxd[buf][part * PART + k][q], acc[q]);
        acc2[q] = fma(tv[k + 1], sxd[buf][part * PART + k + 1][q], acc2[q]);
      }
  }
#pragma unroll
  for (int q = 0; q < NR; q++) sacc[part][row][q] = acc[q] + acc2[q];
  __syncthreads();
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    T t = T(0);
#pragma unroll
    for (int p = 0; p < NQ; p++) t += sacc[p][rr][q];
    sb[rr][q] -= t;
  }
  __syncthreads();
  // 3. x = inv(T_bb) b: thread (row, part) sums over a quarter of the columns
  {
    T v[NR], v2[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) v[q] = v2[q] = T(0);
#pragma unroll
    for (int c = part * PART; c < part * PART + PART; c += 2) {
      const T w = sW[row][c], w2 = sW[row][c + 1];
#pragma unroll
      for (int q = 0; q < NR; q++) {
        v[q] = fma(w, sb[c][q], v[q]);
        v2[q] = fma(w2, sb[c + 1][q], v2[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < NR; q++) sacc[part][row][q] = v[q] + v2[q];
  }
  __syncthreads();
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    T t = T(0);
#pragma unroll
    for (int p = 0; p < NQ; p++) t += sacc[p][rr][q];
    if (rr < rows && q < nrhs) {
      X[r0 + rr + (long)q * ldx] = t;
      if constexpr (sizeof(T) == 4)
        xt[(long)(r0 + rr) * NR + q] =
            ((unsigned long long)(unsigned)epoch << 32) | (unsigned long long)__float_as_uint((float)t);
    }
  }
  __syncthreads();
  if (tid == 0) {  // the barrier orders every thread's x stores before this release
    __threadfence();
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + bi), "r"(epoch) : "memory");
  }
}

// The 128 x 128 diagonal blocks' inverses from the 64 x 64 ones (W64, as
// trinv_kernel leaves them): lower [W0 0; -W1 T10 W0  W1], upper
// [W0  -W0 T01 W1; 0 W1], with W1 = I when the last block has one sub-block.
// One CTA per block, the 128 x 128 block in shared memory: the off-diagonal
// quadrant first holds T's, then Y = T10 W0 (or T01 W1), then -W1 Y (or
// -W0 Y).  Written column-major, 128 x 128 per block.
template <typename T>
__global__ void __launch_bounds__(256)
trinv128_kernel(int n, const T *__restrict__ Tp, long tr, long tc, int lower, const T *__restrict__ W64,
                T *__restrict__ W128) {
  extern __shared__ __align__(16) unsigned char t128_smem[];
  T(*s)[CB + 1] = reinterpret_cast<T(*)[CB + 1]>(t128_smem);
  const int b = blockIdx.x, r0 = b * CB, tid = threadIdx.x;
  const int nsub = min(2, (n - r0 + BS - 1) / BS);
  for (int base = tid; base < CB * CB; base += 8 * 256) {  // eight loads in flight per thread
    T v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int idx = base + 256 * q;
      const int i = idx % CB, k = idx / CB, qi = i / BS, qk = k / BS, ii = i % BS, kk = k % BS;
      v[q] = T(0);
      if (qi == qk) {
        if (qi < nsub) v[q] = W64[(long)(2 * b + qi) * BS * BS + ii + kk * BS];
        else v[q] = ii == kk ? T(1) : T(0);
      } else if (lower ? qi == 1 : qi == 0) {  // the triangle's off-diagonal quadrant
        const int gi = r0 + i, gk = r0 + k;
        if (gi < n && gk < n) v[q] = Tp[gi * tr + gk * tc];
      }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) s[(base + 256 * q) % CB][(base + 256 * q) / CB] = v[q];
  }
  __syncthreads();
  // off-diagonal quadrant at (oi, ok); the products read the diagonal
  // quadrants at (ok, ok) (first) and (oi, oi) (second)
  const int oi = lower ? BS : 0, ok = lower ? 0 : BS;
  T y[BS * BS / 256];
#pragma unroll
  for (int e = 0; e < BS * BS / 256; e++) {
    const int idx = tid + 256 * e, i = idx % BS, j = idx / BS;
    T acc = T(0);
#pragma unroll 16
    for (int k = 0; k < BS; k++) acc = fma(s[oi + i][ok + k], s[ok + k][ok + j], acc);
    y[e] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < BS * BS / 256; e++) {
    const int idx = tid + 256 * e;
    s[oi + idx % BS][ok + idx / BS] = y[e];
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < BS * BS / 256; e++) {
    const int idx = tid + 256 * e, i = idx % BS, j = idx / BS;
    T acc = T(0);
#pragma unroll 16
    for (int k = 0; k < BS; k++) acc = fma(s[oi + i][oi + k], s[oi + k][ok + j], acc);
    y[e] = -acc;
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < BS * BS / 256; e++) {
    const int idx = tid + 256 * e;
    s[oi + idx % BS][ok + idx / BS] = y[e];
  }
  __syncthreads();
  T *Wb = W128 + (long)b * CB * CB;
  for (int idx = tid; idx < CB * CB; idx += 256) Wb[idx] = s[idx % CB][idx / CB];
}

}  // namespace

size_t trsv_w_elems(int n) { return (size_t)cdiv(n, CB) * CB * CB + (size_t)cdiv(n, BS) * BS * BS; }

// Inverted 128 x 128 diagonal blocks of op(A)'s triangle, as trsv_w_dev takes
// them (W holds trsv_w_elems(n) elements: the 128 x 128 inverses, then the
// 64 x 64 ones they are assembled from).
template <typename T>
void trsv_inverse_dev(int uplo, int trans, int diag, int n, const T *A, long lda, T *W, cudaStream_t st) {
  if (n <= 0) return;
  const bool tr = trans != kNoTrans;
  const long tstr = tr ? lda : 1, tcol = tr ? 1 : lda;
  const int lower = (uplo == kLower) != tr;
  T *W64 = W + (size_t)cdiv(n, CB) * CB * CB;
  trinv_dev<T>(n, A, tstr, tcol, lower, diag == kUnit, W64, st);
  constexpr int smem = CB * (CB + 1) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trinv128_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  trinv128_kernel<T><<<cdiv(n, CB), 256, smem, st>>>(n, A, tstr, tcol, lower, W64, W);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trsv_inverse_dev<double>(int, int, int, int, const double *, long, double *, cudaStream_t);
template void trsv_inverse_dev<float>(int, int, int, int, const float *, long, float *, cudaStream_t);

// Solve op(A) X = B in place (Left side only): the inverted diagonal blocks
// once, then one launch per 8 right-hand sides.
template <typename T>
void trsv_dev(int uplo, int trans, int diag, int n, int nrhs, const T *A, long lda, T *B, long ldb,
              cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return;
  T *W = (T *)scratch(kSlotTrsmW, sizeof(T) * trsv_w_elems(n));
  trsv_inverse_dev<T>(uplo, trans, diag, n, A, lda, W, st);
  for (int c0 = 0; c0 < nrhs; c0 += 8)
    trsv_w_dev<T>(uplo, trans, n, std::min(8, nrhs - c0), A, lda, W, B + (long)c0 * ldb, ldb, st);
}
template void trsv_dev<double>(int, int, int, int, int, const double *, long, double *, long, cudaStream_t);
template void trsv_dev<float>(int, int, int, int, int, const float *, long, float *, long, cudaStream_t);

// The same solve with the inverted diagonal blocks W already computed
// (trsv_inverse_dev): for repeated solves with one factor.
template <typename T>
void trsv_w_dev(int uplo, int trans, int n, int nrhs, const T *A, long lda, const T *W, T *B, long ldb,
                cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return;
  const bool tr = trans != kNoTrans;
  const long tstr = tr ? lda : 1, tcol = tr ? 1 : lda;  // effective T(i,k) = A[i*tstr + k*tcol]
  const int lower = (uplo == kLower) != tr;
  const int nb = cdiv(n, CB);
  // workspace: ticket counter, error word, flags, and (FP32) the tagged copy
  // of x, 8 words per row
  const size_t nctl = (size_t)cdiv(nb + 64, 2) * 2, ntag = sizeof(T) == 4 ? (size_t)nb * CB * 8 : 0;
  int *ctl = (int *)scratch(kSlotTrsvCtl, sizeof(int) * nctl + sizeof(unsigned long long) * ntag);
  const int epoch = 1;
  int *counter = ctl, *err = ctl + 1, *flags = ctl + 64;
  unsigned long long *xt = (unsigned long long *)(ctl + nctl);
  ATLB_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(int) * nctl + sizeof(unsigned long long) * ntag, st));
  // sW, sxd, sb, sacc (trsv_kernel's layout), for the largest NR
  constexpr int smem = (CB * (CB + 1) + (2 * CB + CB + NQ * CB) * 8) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  if (nrhs == 1)
    trsv_kernel<T, 1><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err, xt);
  else if (nrhs <= 4)
    trsv_kernel<T, 4><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err, xt);
  else
    trsv_kernel<T, 8><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err, xt);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trsv_w_dev<double>(int, int, int, int, const double *, long, const double *, double *, long,
                                 cudaStream_t);
template void trsv_w_dev<float>(int, int, int, int, const float *, long, const float *, float *, long,
                                cudaStream_t);

}  // namespace atlb
