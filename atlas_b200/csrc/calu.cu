// Tournament-pivoting ("communication-avoiding", CALU) leaf panel for the
// FP32 factorization inside the mixed-precision solvers.
//
// Method: Grigori, Demmel & Xiang, "CALU: a communication optimal LU
// factorization algorithm", SIAM J. Matrix Anal. Appl. 32(4), 2011 (TSLU with
// a flat reduction tree).  The pivots differ from partial pivoting's; only
// the solvers' FP64 refinement sees the factors, so ATLAS's pivot order
// (which the FP64 getrf keeps) is not needed here, and in exchange a 32-column
// panel needs no exchange between CTAs per column:
//
//   A. every CTA of the cluster runs partial pivoting on its own 512 rows
//      (CTA-local steps) and keeps the original values of the <= 32 rows it
//      chose as its candidates;
//   B. every CTA reads all CTAs' candidates over distributed shared memory
//      and runs partial pivoting on them -- the same computation on the same
//      data in every CTA, so all CTAs agree on the panel's pivot rows and on
//      their L11 multipliers and U11 rows without another exchange;
//   C. every other row solves l U11 = (its original row) for its multipliers,
//      and rows are written at their final positions (LAPACK's interchange
//      sequence, ipiv);
//   D. the block's other columns of the rows that moved are interchanged and
//      U12 = L11^-1 A12 is solved, each CTA on its own share of columns.
//
// Layout: a CTA has 128 threads, each holding 4 rows (rows t, t+128, t+256,
// t+384 of the CTA's 512) in registers, "shifted": register 0 is always the
// current column, and the multiplier of each step enters at the end, so after
// step j a row holds its remaining columns followed by its j multipliers.  A
// pivot step is one warp arg-max (integer keys), one __syncthreads, a CTA
// arg-max over the four warps' winners, and a rank-1 update with the winner's
// row read from shared memory once per thread for its four rows (reading it
// once per row is what bounds a one-row-per-thread step: 512 threads x 128 B
// of broadcast loads per column).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <cooperative_groups.h>
#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace atlb {
namespace {

constexpr int CT = 128;              // threads per CTA
constexpr int CR = 4;                // rows per thread
constexpr int CROWS = CT * CR;       // rows per CTA
constexpr int CNB = 32;              // panel width
constexpr int CW = CT / 32;          // warps per CTA
constexpr int kCaluMaxCluster = 16;
constexpr int OLD = CNB + 1;         // row stride of the original rows in shared memory

// |v| as an ordered integer key + 1 (0 = no candidate; NaN never wins)
__device__ __forceinline__ unsigned calu_key(float v) {
  const float t = fabsf(v);
  return t >= 0.f ? __float_as_uint(t) + 1u : 1u;
}

__device__ __forceinline__ void calu_cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void calu_cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

struct CaluShared {
  float rowbuf[2][CW][CNB];          // the warps' winners (masked rows), by step parity
  unsigned wkey[2][CW];
  int wrid[2][CW];
  float cand[CNB][CNB];              // this CTA's candidate rows (original values)
  int candrow[CNB];                  // ... and their panel rows
  float rec[CNB][CNB];               // step j's winner row: U(j, j..) then its multipliers
  int win[CNB];                      // panel row of pivot j
  float Ush[CNB][CNB];               // U(j, j + k) at [j][k] (zero past the row)
  float U11[CNB][CNB + 1];
  float L11[CNB][CNB + 1];
  float urcp[CNB];
  int e_row[2 * CNB], e_pos[2 * CNB];  // rows that move: panel row -> final position
  int ne, nloc;
  float stage[2 * CNB][16];          // phase D: moved rows of up to 16 columns
};

// One partial-pivoting step over the thread's rows (see the file comment).
// Returns the winner's row id (-1: no active row left anywhere in the CTA).
// RECORD: the winner stores its whole register row in S.rec[j].
template <bool RECORD>
__device__ __forceinline__ int calu_step(int j, float (&a)[CR][CNB], const int (&rid)[CR], bool (&act)[CR],
                                         CaluShared &S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, b = j & 1;
  unsigned best = 0;
  int bq = 0;
#pragma unroll
  for (int q = 0; q < CR; q++) {
    const unsigned key = act[q] ? calu_key(a[q][0]) : 0u;
    if (key > best) { best = key; bq = q; }
  }
  const unsigned mk = __reduce_max_sync(0xffffffffu, best);
  const int wl = __ffs(__ballot_sync(0xffffffffu, best == mk)) - 1;
  if (lane == wl) {
    // the row without its multipliers (registers >= CNB - j hold them)
    float4 *dst = reinterpret_cast<float4 *>(S.rowbuf[b][warp]);
#pragma unroll
    for (int q = 0; q < CR; q++) {
      if (q == bq) {
#pragma unroll
        for (int k4 = 0; k4 < CNB / 4; k4++) {
          float4 v;
          v.x = 4 * k4 + 0 < CNB - j ? a[q][4 * k4 + 0] : 0.f;
          v.y = 4 * k4 + 1 < CNB - j ? a[q][4 * k4 + 1] : 0.f;
          v.z = 4 * k4 + 2 < CNB - j ? a[q][4 * k4 + 2] : 0.f;
          v.w = 4 * k4 + 3 < CNB - j ? a[q][4 * k4 + 3] : 0.f;
          dst[k4] = v;
        }
      }
    }
    int r = -1;
#pragma unroll
    for (int q = 0; q < CR; q++)
      if (q == bq) r = rid[q];
    S.wkey[b][warp] = mk;
    S.wrid[b][warp] = mk ? r : -1;
  }
  __syncthreads();
  const unsigned k2 = lane < CW ? S.wkey[b][lane] : 0u;
  const unsigned m2 = __reduce_max_sync(0xffffffffu, k2);
  if (m2 == 0u) return -1;  // uniform: no active row in the CTA
  const int cw = __ffs(__ballot_sync(0xffffffffu, lane < CW && k2 == m2)) - 1;
  const int prow = S.wrid[b][cw];
  const float4 *u4 = reinterpret_cast<const float4 *>(S.rowbuf[b][cw]);
  const float4 h = u4[0];
  const float rcp = h.x != 0.f ? 1.f / h.x : 0.f;
#pragma unroll
  for (int q = 0; q < CR; q++) {
    if (!act[q]) continue;
    if (rid[q] == prow) {
      act[q] = false;
      if (RECORD) {
        float4 *dst = reinterpret_cast<float4 *>(S.rec[j]);
#pragma unroll
        for (int k4 = 0; k4 < CNB / 4; k4++)
          dst[k4] = make_float4(a[q][4 * k4], a[q][4 * k4 + 1], a[q][4 * k4 + 2], a[q][4 * k4 + 3]);
      }
      continue;
    }
    const float l = a[q][0] * rcp;
    a[q][0] = fmaf(-l, h.y, a[q][1]);  // the next column first: it decides the next pivot
    a[q][1] = fmaf(-l, h.z, a[q][2]);
    a[q][2] = fmaf(-l, h.w, a[q][3]);
#pragma unroll
    for (int k4 = 1; k4 < CNB / 4; k4++) {
      const float4 v = u4[k4];
      a[q][4 * k4 - 1] = fmaf(-l, v.x, a[q][4 * k4]);
      a[q][4 * k4] = fmaf(-l, v.y, a[q][4 * k4 + 1]);
      a[q][4 * k4 + 1] = fmaf(-l, v.z, a[q][4 * k4 + 2]);
      a[q][4 * k4 + 2] = fmaf(-l, v.w, a[q][4 * k4 + 3]);
    }
    a[q][CNB - 1] = l;
  }
  return prow;
}

__device__ int g_calu_bad_args = 0;  // set if a launch ever received an impossible shape

// The panel of M x ncols (ncols <= 32) at A; ipiv + roff numbering; the block's
// nleft columns left of the panel and nright right of it get the interchanges,
// the right ones also U12 = L11^-1 A12.
__global__ void __launch_bounds__(CT, 1)
getf2_calu_kernel(int M, int ncols, float *__restrict__ A, long lda, int *__restrict__ ipiv, int roff,
                  int *__restrict__ dinfo, int nleft, int nright) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), crank = (int)cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int MN = min(M, ncols);
  extern __shared__ __align__(16) unsigned char calu_dyn[];
  float *orig = reinterpret_cast<float *>(calu_dyn);  // [CROWS][OLD]
  __shared__ __align__(16) CaluShared S;
  if (ncols > CNB || ncols < 1 || C * CROWS < M || nleft + nright > 256) {
    if (tid == 0) atomicExch(&g_calu_bad_args, 1);
    calu_cluster_arrive();  // every CTA takes this branch alike: keep the cluster barriers paired
    calu_cluster_wait();
    return;
  }
  const int base = crank * CROWS;
  const int rows_here = max(0, min(CROWS, M - base));

  // ---- load the CTA's rows (coalesced: thread t takes rows t + 128 q)
  float a[CR][CNB];
  int rid[CR];
  bool act[CR];
#pragma unroll
  for (int q = 0; q < CR; q++) {
    const int lr = tid + CT * q;
    rid[q] = base + lr;
    act[q] = lr < rows_here;
    const float *src = A + (act[q] ? rid[q] : 0);
#pragma unroll
    for (int k = 0; k < CNB; k++) a[q][k] = (act[q] && k < ncols) ? __ldg(src + (long)k * lda) : 0.f;
#pragma unroll
    for (int k = 0; k < CNB; k++) orig[lr * OLD + k] = a[q][k];
  }
  __syncthreads();

  // ---- A. local candidates
  const int nloc = min(MN, rows_here);
  for (int j = 0; j < nloc; j++) {
    const int p = calu_step<false>(j, a, rid, act, S);
    if (tid == 0) S.candrow[j] = p;
  }
  __syncthreads();
  for (int e = tid; e < nloc * CNB; e += CT) {
    const int j = e / CNB, k = e - j * CNB, lr = S.candrow[j] - base;
    S.cand[j][k] = lr >= 0 && lr < rows_here ? orig[lr * OLD + k] : 0.f;
  }
  if (tid == 0) S.nloc = nloc;
  __syncwarp();
  calu_cluster_arrive();  // candidates are out
  calu_cluster_wait();

  // ---- B. the merge, in every CTA: candidate g = c * MN + j (CTA c's j-th)
#pragma unroll
  for (int q = 0; q < CR; q++) {
    const int g = tid + CT * q, c = g / max(MN, 1), j = g - c * MN;
    bool valid = c < C && MN > 0;
    int nc = 0;
    if (valid) {
      nc = min(MN, max(0, min(CROWS, M - c * CROWS)));
      valid = j < nc;
    }
    act[q] = valid;
    rid[q] = -1;
    if (valid) {
      const CaluShared *R = cl.map_shared_rank(&S, c);
      const float4 *src = reinterpret_cast<const float4 *>(R->cand[j]);
#pragma unroll
      for (int k4 = 0; k4 < CNB / 4; k4++) {
        const float4 v = src[k4];
        a[q][4 * k4] = v.x;
        a[q][4 * k4 + 1] = v.y;
        a[q][4 * k4 + 2] = v.z;
        a[q][4 * k4 + 3] = v.w;
      }
      rid[q] = R->candrow[j];
    } else {
#pragma unroll
      for (int k = 0; k < CNB; k++) a[q][k] = 0.f;
    }
  }
  // no remote read follows: the barrier's wait is the last thing before exit,
  // so no CTA leaves while another still reads its candidates
  calu_cluster_arrive();
  for (int j = 0; j < MN; j++) {
    const int p = calu_step<true>(j, a, rid, act, S);
    if (tid == 0) S.win[j] = p;
  }
  __syncthreads();

  // ---- C. L11, U11, the interchanges, the multipliers of every row
  for (int e = tid; e < CNB * CNB; e += CT) {
    const int j = e / CNB, m = e - j * CNB;
    const float v = j < MN ? S.rec[j][m] : 0.f;
    if (m < CNB - j) {  // U(j, j + m)
      const float u = j + m < ncols ? v : 0.f;
      S.U11[j][j + m] = u;
      S.Ush[j][m] = u;
    } else {            // multiplier l_i of row j, i = m - (CNB - j) < j
      S.L11[j][m - (CNB - j)] = v;
      S.Ush[j][m] = 0.f;
    }
    if (m < j) S.U11[j][m] = 0.f;
    if (m >= j) S.L11[j][m] = m == j ? 1.f : 0.f;
  }
  __syncthreads();
  if (tid < CNB) {
    const float d = tid < MN ? S.U11[tid][tid] : 1.f;
    S.urcp[tid] = d != 0.f ? 1.f / d : 0.f;
    if (crank == 0 && tid < MN && d == 0.f) atomicMin(dinfo, roff + tid + 1);
  }
  if (warp == 0) {
    // LAPACK's interchange sequence: at step j swap positions j and (position of win[j])
    if (lane == 0) {
      int ne = 0;
      for (int i = 0; i < MN; i++) { S.e_row[ne] = i; S.e_pos[ne] = i; ne++; }
      for (int j = 0; j < MN; j++)
        if (S.win[j] >= MN) { S.e_row[ne] = S.win[j]; S.e_pos[ne] = S.win[j]; ne++; }
      S.ne = ne;
    }
    __syncwarp();
    const int ne = S.ne;
    int er0 = lane < ne ? S.e_row[lane] : -1, ep0 = lane < ne ? S.e_pos[lane] : -1;
    int er1 = lane + 32 < ne ? S.e_row[lane + 32] : -1, ep1 = lane + 32 < ne ? S.e_pos[lane + 32] : -1;
    for (int j = 0; j < MN; j++) {
      const int pr = S.win[j];
      const unsigned m0 = __ballot_sync(0xffffffffu, er0 == pr), m1 = __ballot_sync(0xffffffffu, er1 == pr);
      const int p = m0 ? __shfl_sync(0xffffffffu, ep0, __ffs(m0) - 1)
                       : __shfl_sync(0xffffffffu, ep1, m1 ? __ffs(m1) - 1 : 0);
      if (lane == 0 && crank == 0) ipiv[j] = roff + p;
      // positions j and p exchange their rows
      const bool a0 = ep0 == j, b0 = ep0 == p, a1 = ep1 == j, b1 = ep1 == p;
      if (a0) ep0 = p; else if (b0) ep0 = j;
      if (a1) ep1 = p; else if (b1) ep1 = j;
    }
    if (lane < ne) S.e_pos[lane] = ep0;
    if (lane + 32 < ne) S.e_pos[lane + 32] = ep1;
  }
  __syncthreads();
  const int ne = S.ne;
  // each of this thread's rows: its panel values at its final position
  int fpos[CR], pj[CR];
#pragma unroll
  for (int q = 0; q < CR; q++) {
    const int lr = tid + CT * q, r = base + lr;
    fpos[q] = r;
    pj[q] = -1;
    for (int e = 0; e < ne; e++)
      if (S.e_row[e] == r) fpos[q] = S.e_pos[e];
    for (int j = 0; j < MN; j++)
      if (S.win[j] == r) pj[q] = j;
#pragma unroll
    for (int k = 0; k < CNB; k++) a[q][k] = lr < rows_here ? orig[lr * OLD + k] : 0.f;
  }
  // l U11 = o by forward substitution over U11's rows, shifted like the pivot
  // steps (the current column is register 0, each multiplier enters at the
  // end): after CNB steps a[q][k] = l_k.  Rows of U11 past MN are zero with a
  // unit reciprocal, so the padding columns give zero multipliers.
#pragma unroll 1
  for (int i = 0; i < CNB; i++) {
    const float4 *u4 = reinterpret_cast<const float4 *>(S.Ush[i]);
    const float ri = S.urcp[i];
    const float4 h = u4[0];
#pragma unroll
    for (int q = 0; q < CR; q++) {
      const float li = a[q][0] * ri;
      a[q][0] = fmaf(-li, h.y, a[q][1]);
      a[q][1] = fmaf(-li, h.z, a[q][2]);
      a[q][2] = fmaf(-li, h.w, a[q][3]);
#pragma unroll
      for (int k4 = 1; k4 < CNB / 4; k4++) {
        const float4 v = u4[k4];
        a[q][4 * k4 - 1] = fmaf(-li, v.x, a[q][4 * k4]);
        a[q][4 * k4] = fmaf(-li, v.y, a[q][4 * k4 + 1]);
        a[q][4 * k4 + 1] = fmaf(-li, v.z, a[q][4 * k4 + 2]);
        a[q][4 * k4 + 2] = fmaf(-li, v.w, a[q][4 * k4 + 3]);
      }
      a[q][CNB - 1] = li;
    }
  }
#pragma unroll
  for (int q = 0; q < CR; q++) {
    const int lr = tid + CT * q;
    if (lr >= rows_here) continue;
    float *dst = A + fpos[q];
    if (pj[q] >= 0) {
      const int j = pj[q];
      for (int k = 0; k < ncols; k++) dst[(long)k * lda] = k < j ? S.L11[j][k] : S.U11[j][k];
    } else {
#pragma unroll
      for (int k = 0; k < CNB; k++)
        if (k < ncols) dst[(long)k * lda] = a[q][k];
    }
  }

  // ---- D. the block's other columns: CTA c takes columns c, c + C, ...
  const int nother = nleft + nright;
  if (nother > 0) {
    int nm = 0;
    __shared__ int m_from[2 * CNB], m_to[2 * CNB];
    if (tid == 0) {
      for (int e = 0; e < ne; e++)
        if (S.e_pos[e] != S.e_row[e]) { m_from[nm] = S.e_row[e]; m_to[nm] = S.e_pos[e]; nm++; }
      S.nloc = nm;
    }
    __syncthreads();
    nm = S.nloc;
    for (int c0 = crank; c0 < nother; c0 += 16 * C) {
      // up to 16 of this CTA's columns at a time: c0 + C * s, s < 16
      for (int e = tid; e < nm * 16; e += CT) {
        const int i = e % nm, s = e / nm, c = c0 + C * s;
        if (c < nother) {
          const int col = c < nleft ? c - nleft : ncols + (c - nleft);
          S.stage[i][s] = __ldcg(A + m_from[i] + (long)col * lda);
        }
      }
      __syncthreads();
      for (int e = tid; e < nm * 16; e += CT) {
        const int i = e % nm, s = e / nm, c = c0 + C * s;
        if (c < nother) {
          const int col = c < nleft ? c - nleft : ncols + (c - nleft);
          A[m_to[i] + (long)col * lda] = S.stage[i][s];
        }
      }
      __syncthreads();
      // U12 = L11^-1 A12 on this CTA's right columns: one warp per column,
      // lane = row, forward substitution by shuffles
      if (MN > 1) {
        for (int s = warp; s < 16; s += CW) {
          const int c = c0 + C * s;
          if (c >= nother || c < nleft) continue;
          float *col = A + (long)(ncols + (c - nleft)) * lda;
          float x = lane < MN ? __ldcg(col + lane) : 0.f;
          for (int k = 0; k < MN - 1; k++) {
            const float xk = __shfl_sync(0xffffffffu, x, k);
            if (lane > k) x = fmaf(-S.L11[lane][k], xk, x);
          }
          if (lane < MN) col[lane] = x;
        }
      }
      __syncthreads();
    }
  }
  calu_cluster_wait();
}

int g_calu_cluster = -1;

int calu_smem_bytes() { return CROWS * OLD * (int)sizeof(float); }

// Largest cluster (<= 16) of the kernel the device co-schedules; 0 when none.
int calu_max_cluster() {
  if (g_calu_cluster >= 0) return g_calu_cluster;
  g_calu_cluster = 0;
  auto kern = getf2_calu_kernel;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, calu_smem_bytes()) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int c : {kCaluMaxCluster, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c, 1, 1);
    cfg.blockDim = dim3(CT, 1, 1);
    cfg.dynamicSmemBytes = calu_smem_bytes();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) { cudaGetLastError(); n = 0; }
    if (n > 0) { g_calu_cluster = c; break; }
  }
  return g_calu_cluster;
}

}  // namespace

int calu_max_rows() { return calu_max_cluster() * CROWS; }

bool launch_calu_panel(int M, int ncols, float *A, long lda, int *ipiv, int roff, int *dinfo, int nleft,
                       int nright, cudaStream_t st) {
  if (ncols > CNB || ncols < 1 || nleft + nright > 256 || M < 1) return false;
  const int C = cdiv(M, CROWS);
  if (C > calu_max_cluster()) return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(CT, 1, 1);
  cfg.dynamicSmemBytes = calu_smem_bytes();
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATLB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, getf2_calu_kernel, M, ncols, A, lda, ipiv, roff, dinfo, nleft,
                                     nright));
  return true;
}

}  // namespace atlb
