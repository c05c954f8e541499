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
// already in registers.  The two sub-blocks are then solved in turn with
// the inverted 64x64 diagonal blocks (trinv_kernel's W) and the block is
// published.  Every wait on a flag is bounded: after ~1 s the kernel records
// an error in *err and stops waiting (the result is then wrong but the GPU
// is released).  The launcher clears the ticket counter and the flags before
// each launch.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int BS = 64;       // rows of a diagonal block (W's blocks)
constexpr int CB = 2 * BS;   // rows of one CTA's block
constexpr int TT = 256;      // threads: two per row of the CTA's block

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
            const T *__restrict__ W, T *X, long ldx, int *counter, int *flags, int epoch, int *err) {
  extern __shared__ __align__(16) unsigned char trsv_smem[];
  T(*sW)[BS][BS + 1] = reinterpret_cast<T(*)[BS][BS + 1]>(trsv_smem);  // the two inverted diagonal blocks
  T(*sxd)[CB][NR] = reinterpret_cast<T(*)[CB][NR]>(sW + 2);             // x of a solved block, double-buffered
  T(*sb)[NR] = reinterpret_cast<T(*)[NR]>(sxd + 2);                     // this block's b, then its x
  T(*spart)[BS][NR] = reinterpret_cast<T(*)[BS][NR]>(sb + CB);          // [4]: quarter sums
  T(*sacc)[CB][NR] = reinterpret_cast<T(*)[CB][NR]>(spart + 4);         // [2]: the two halves' sums
  __shared__ int s_bi, s_ready;
  const int tid = threadIdx.x, lane = tid & 31, nb = (n + CB - 1) / CB;
  if (tid == 0) {
    const int t = atomicAdd(counter, 1);
    s_bi = lower ? t : nb - 1 - t;
  }
  __syncthreads();
  const int bi = s_bi, r0 = bi * CB, rows = min(CB, n - r0);
  const int nsub = (rows + BS - 1) / BS;  // 1 or 2 sub-blocks
  // everything that does not depend on other blocks is fetched first
  for (int sbk = 0; sbk < nsub; sbk++) {
    const T *Wb = W + (long)(r0 / BS + sbk) * BS * BS;
    for (int idx = tid; idx < BS * BS; idx += TT) sW[sbk][idx % BS][idx / BS] = Wb[idx];
  }
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    sb[rr][q] = (rr < rows && q < nrhs) ? X[r0 + rr + (long)q * ldx] : T(0);
  }
  // thread (row, half): row of this block, columns half*64 .. +63 of every solved block
  const int row = tid % CB, half = tid / CB;
  const T *trow = Tp + (long)(r0 + row) * tr;
  const int ndep = lower ? bi : nb - 1 - bi;
  T acc[NR];
#pragma unroll
  for (int q = 0; q < NR; q++) acc[q] = T(0);
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
      load_x(bj, buf);
      __syncthreads();
      const int c0 = bj * CB + half * BS, cols = min(BS, n - c0);
      if (row < rows) {
        const T(*xs)[NR] = sxd[buf] + half * BS;
#pragma unroll 16
        for (int k = 0; k < BS; k++) {
          const T tv = k < cols ? trow[(long)(c0 + k) * tc] : T(0);
#pragma unroll
          for (int q = 0; q < NR; q++) acc[q] = fma(tv, xs[k][q], acc[q]);
        }
      }
      buf ^= 1;
    }
    __syncthreads();  // s_ready is read by every thread before it is rewritten
  }
  // 2. the block just before this one: its matrix values first, then the wait
  if (ndep > 0) {
    const int bj = lower ? ndep - 1 : nb - ndep;
    const int c0 = bj * CB + half * BS, cols = min(BS, n - c0);
    T tv[BS];
#pragma unroll
    for (int k = 0; k < BS; k++) tv[k] = (row < rows && k < cols) ? trow[(long)(c0 + k) * tc] : T(0);
    if (tid == 0) wait_flag(bj);
    __syncthreads();
    load_x(bj, buf);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BS; k++)
#pragma unroll
      for (int q = 0; q < NR; q++) acc[q] = fma(tv[k], sxd[buf][half * BS + k][q], acc[q]);
  }
#pragma unroll
  for (int q = 0; q < NR; q++) sacc[half][row][q] = acc[q];
  __syncthreads();
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    sb[rr][q] -= sacc[0][rr][q] + sacc[1][rr][q];
  }
  __syncthreads();
  // 3. the two sub-blocks in turn (lower: top first): x_s = W_s b_s, then
  // the other sub-block's b -= T(other, s) x_s
  const int i64 = tid % BS, part = tid / BS;  // row of a sub-block, quarter of its columns
  for (int step = 0; step < nsub; step++) {
    const int sbk = lower ? step : nsub - 1 - step;
#pragma unroll
    for (int q = 0; q < NR; q++) {
      T v = T(0);
#pragma unroll
      for (int c = 16 * part; c < 16 * part + 16; c++) v = fma(sW[sbk][i64][c], sb[sbk * BS + c][q], v);
      spart[part][i64][q] = v;
    }
    __syncthreads();
    for (int idx = tid; idx < BS * NR; idx += TT) {
      const int rr = idx % BS, q = idx / BS;
      sb[sbk * BS + rr][q] = (spart[0][rr][q] + spart[1][rr][q]) + (spart[2][rr][q] + spart[3][rr][q]);
    }
    __syncthreads();
    if (step + 1 < nsub) {
      const int oth = 1 - sbk;
      // rows of sub-block oth, columns of sub-block sbk
      const int gr = r0 + oth * BS + i64;
      T v[NR];
#pragma unroll
      for (int q = 0; q < NR; q++) v[q] = T(0);
      if (oth * BS + i64 < rows) {
        const T *tr2 = Tp + (long)gr * tr;
#pragma unroll
        for (int c = 16 * part; c < 16 * part + 16; c++) {
          const int gc = r0 + sbk * BS + c;  // a column of sub-block sbk (past n when it is the partial last one)
          const T tv2 = gc < n ? tr2[(long)gc * tc] : T(0);
#pragma unroll
          for (int q = 0; q < NR; q++) v[q] = fma(tv2, sb[sbk * BS + c][q], v[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < NR; q++) spart[part][i64][q] = v[q];
      __syncthreads();
      for (int idx = tid; idx < BS * NR; idx += TT) {
        const int rr = idx % BS, q = idx / BS;
        sb[oth * BS + rr][q] -= (spart[0][rr][q] + spart[1][rr][q]) + (spart[2][rr][q] + spart[3][rr][q]);
      }
      __syncthreads();
    }
  }
  for (int idx = tid; idx < CB * NR; idx += TT) {
    const int rr = idx % CB, q = idx / CB;
    if (rr < rows && q < nrhs) X[r0 + rr + (long)q * ldx] = sb[rr][q];
  }
  __syncthreads();
  if (tid == 0) {  // the barrier orders every thread's x stores before this release
    __threadfence();
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + bi), "r"(epoch) : "memory");
  }
}

}  // namespace

// Inverted 64x64 diagonal blocks of op(A)'s triangle, as trsv_w_dev takes them.
template <typename T>
void trsv_inverse_dev(int uplo, int trans, int diag, int n, const T *A, long lda, T *W, cudaStream_t st) {
  if (n <= 0) return;
  const bool tr = trans != kNoTrans;
  const long tstr = tr ? lda : 1, tcol = tr ? 1 : lda;
  const int lower = (uplo == kLower) != tr;
  trinv_dev<T>(n, A, tstr, tcol, lower, diag == kUnit, W, st);
}
template void trsv_inverse_dev<double>(int, int, int, int, const double *, long, double *, cudaStream_t);
template void trsv_inverse_dev<float>(int, int, int, int, const float *, long, float *, cudaStream_t);

// Solve op(A) X = B in place for nrhs <= 8 right-hand sides (Left side only).
template <typename T>
void trsv_dev(int uplo, int trans, int diag, int n, int nrhs, const T *A, long lda, T *B, long ldb,
              cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return;
  T *W = (T *)scratch(kSlotTrsmW, sizeof(T) * (size_t)cdiv(n, BS) * BS * BS);
  trsv_inverse_dev<T>(uplo, trans, diag, n, A, lda, W, st);
  trsv_w_dev<T>(uplo, trans, n, nrhs, A, lda, W, B, ldb, st);
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
  // workspace: ticket counter, error word, flags
  int *ctl = (int *)scratch(kSlotTrsvCtl, sizeof(int) * (nb + 64));
  const int epoch = 1;
  int *counter = ctl, *err = ctl + 1, *flags = ctl + 64;
  ATLB_CUDA_CHECK(cudaMemsetAsync(ctl, 0, sizeof(int) * (nb + 64), st));  // counter, flags
  // sW, sxd, sb, spart, sacc (trsv_kernel's layout), for the largest NR
  constexpr int smem = (2 * BS * (BS + 1) + (2 * CB + CB + 4 * BS + 2 * CB) * 8) * (int)sizeof(T);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(trsv_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  if (nrhs == 1) trsv_kernel<T, 1><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  else if (nrhs <= 4) trsv_kernel<T, 4><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  else trsv_kernel<T, 8><<<nb, TT, smem, st>>>(n, nrhs, A, tstr, tcol, lower, W, B, ldb, counter, flags, epoch, err);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
template void trsv_w_dev<double>(int, int, int, int, const double *, long, const double *, double *, long,
                                 cudaStream_t);
template void trsv_w_dev<float>(int, int, int, int, const float *, long, const float *, float *, long,
                                cudaStream_t);

}  // namespace atlb
