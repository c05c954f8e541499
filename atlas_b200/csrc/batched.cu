// Batched factorizations and solves of many small, uneven-size systems.  No
// counterpart in the reference (ATLAS factors one matrix per call); the
// per-problem arithmetic is that of ATL_potrfL / ATL_getf2 / ATL_potrs /
// ATL_getrs on a single small matrix.
//
// One persistent launch per batch: CTAs pull problem indices from an atomic
// counter over a work list sorted by decreasing size (largest first, so the
// tail of the launch is made of small problems), and each problem is handled
// entirely by one CTA.  Cholesky: orders up to batch_posv_small are factored
// with the whole matrix in shared memory, larger ones (up to 256) in panels
// of batch_posv_pw columns staged in shared memory with the trailing update
// written back to global memory (L2-resident at these sizes).  LU: 16-column
// pivoted panels in shared memory, the trailing update on the FP64 tensor
// cores in global memory.  The solves run in blocks of 16 rows.  Nothing
// waits on another CTA, so the launch cannot stall.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "chol_blocks.cuh"
#include "kernels.h"
#include "staging.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

constexpr int BT = 256;       // threads per CTA
constexpr int MAXN = 256;
// Size buckets of the Cholesky path (tunable, tuning.cu): orders up to
// batch_posv_small are factored whole in shared memory, larger ones in panels
// of batch_posv_pw columns.

struct Prob {
  double *A;
  double *B;
  int *ipiv;
  int n, lda, ldb, nrhs;
};

// dst (rows x cols, ld ldd, shared memory) = src (ld lds, global), eight
// loads in flight per thread before their stores (a plain strided loop would
// wait for each load in turn)
__device__ __forceinline__ void stage_tile(double *dst, int ldd, const double *src, long lds, int rows, int cols) {
  const int tot = rows * cols, tid = threadIdx.x;
  for (int base = 0; base < tot; base += BT * 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * BT + tid;
      v[u] = idx < tot ? src[idx % rows + (long)(idx / rows) * lds] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * BT + tid;
      if (idx < tot) dst[idx % rows + (idx / rows) * ldd] = v[u];
    }
  }
}

// ---------------------------------------------------------------- Cholesky

// Triangular solve of one right-hand side held in shared memory (b, n <=
// MAXN) with T in shared or global memory (ld ldt): op(T) x = b, op(T)
// lower (forward) or upper (backward) triangular, T itself read transposed
// when trans.  Blocks of 16 rows: warp 0 solves a block's 16 x 16 diagonal
// part (x_c by shuffle), then every thread subtracts the block's
// contribution from one remaining row -- two barriers per block instead of
// two per row.
__device__ void tri_solve_smem(const double *T, long ldt, int n, double *b, bool lower, bool unit, bool trans) {
  const int tid = threadIdx.x;
  auto at = [&](int i, int c) { return trans ? T[c + (long)i * ldt] : T[i + (long)c * ldt]; };
  const int nblk = (n + 15) / 16;
  for (int t = 0; t < nblk; t++) {
    const int b0 = lower ? 16 * t : 16 * (nblk - 1 - t), bs = min(16, n - b0);
    if (tid < 32) {
      const int i = tid;
      double x = i < bs ? b[b0 + i] : 0.0;
      if (lower) {
        for (int c = 0; c < bs; c++) {
          if (!unit && i == c) x = x / at(b0 + c, b0 + c);
          const double xc = __shfl_sync(0xffffffffu, x, c);
          if (i > c && i < bs) x = fma(-at(b0 + i, b0 + c), xc, x);
        }
      } else {
        for (int c = bs - 1; c >= 0; c--) {
          if (!unit && i == c) x = x / at(b0 + c, b0 + c);
          const double xc = __shfl_sync(0xffffffffu, x, c);
          if (i < c) x = fma(-at(b0 + i, b0 + c), xc, x);
        }
      }
      if (i < bs) b[b0 + i] = x;
    }
    __syncthreads();
    const int r0 = lower ? b0 + bs : 0, r1 = lower ? n : b0;
    for (int i = r0 + tid; i < r1; i += BT) {
      double acc = b[i];
      for (int c = 0; c < bs; c++) acc = fma(-at(i, b0 + c), b[b0 + c], acc);
      b[i] = acc;
    }
    __syncthreads();
  }
}

// A = L L^T: forward then backward substitution for nrhs columns of B
// (global), L lower in shared or global memory (ld ldl)
__device__ void chol_solve(const double *L, int ldl, int n, double *B, int ldb, int nrhs) {
  __shared__ double sbv[MAXN];
  for (int r = 0; r < nrhs; r++) {
    double *bg = B + (long)r * ldb;
    for (int i = threadIdx.x; i < n; i += BT) sbv[i] = bg[i];
    __syncthreads();
    tri_solve_smem(L, ldl, n, sbv, true, false, false);   // L y = b
    tri_solve_smem(L, ldl, n, sbv, false, false, true);   // L^T x = y
    for (int i = threadIdx.x; i < n; i += BT) bg[i] = sbv[i];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(BT)
batched_posv_kernel(const Prob *__restrict__ probs, const int *__restrict__ order, int count,
                    int *__restrict__ next, int *__restrict__ info, int SMALL, int PW) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_p;
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) {
      const int t = atomicAdd(next, 1);
      s_p = t < count ? order[t] : -1;
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) return;
    const Prob pr = probs[p];
    const int n = pr.n;
    int fail = 0;
    if (n <= SMALL) {
      const int lds = cholb::ld_for(n);
      stage_tile(sm, lds, pr.A, pr.lda, n, n);
      __syncthreads();
      fail = cholb::chol_smem(sm, lds, n);
      for (int idx = tid; idx < n * n; idx += BT) {
        const int i = idx % n, k = idx / n;
        if (i >= k) pr.A[i + (long)k * pr.lda] = sm[i + k * lds];
      }
      __syncthreads();
      if (!fail) chol_solve(sm, lds, n, pr.B, pr.ldb, pr.nrhs);
    } else {
      // panels of PW columns: factor the panel (rows j..n) in shared memory,
      // then update the trailing lower triangle in global memory
      for (int j = 0; j < n && !fail; j += PW) {
        const int jb = min(PW, n - j), m = n - j, lds = cholb::ld_for(m);
        stage_tile(sm, lds, pr.A + j + (long)j * pr.lda, pr.lda, m, jb);
        __syncthreads();
        {
          const int f = cholb::chol_panel(sm, lds, m, jb);
          if (f) fail = j + f;
        }
        for (int idx = tid; idx < m * jb; idx += BT) {
          const int i = idx % m, k = idx / m;
          if (i >= k) pr.A[j + i + (long)(j + k) * pr.lda] = sm[i + k * lds];
        }
        if (fail) break;
        // trailing update: A[j+jb.., j+jb..] -= P2 P2^T (lower), P2 = panel rows jb..m
        if (m > jb) cholb::syrk_panel(m - jb, m - jb, jb, sm + jb, lds, pr.A + (j + jb) + (long)(j + jb) * pr.lda, pr.lda);
        __syncthreads();
      }
      __syncthreads();
      if (!fail) chol_solve(pr.A, pr.lda, n, pr.B, pr.ldb, pr.nrhs);
    }
    if (tid == 0) info[p] = fail;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- LU

// Blocked LU with partial pivoting of one problem by one CTA, the matrix in
// place in global memory (L2-resident at these orders), ATL_getrfC's
// right-looking step on panels of LPW columns:
//   1. the panel (rows j..n-1) is staged in shared memory and factored there
//      column by column: arg-max with the first maximum on ties
//      (cblas_idamax / ATL_getf2), the interchange inside the panel, the
//      scaling (by the reciprocal when the pivot is a normal number), the
//      rank-1 update of the panel's columns right of it;
//   2. the panel goes back, ipiv[j + c] = j + its pivot row;
//   3. the panel's interchanges, composed into one row permutation, move
//      the rows of every column outside the panel (LAPACK's laswp on the
//      left and right parts) in one gather / scatter pass;
//   4. U12 = L11^-1 A12 (one thread per column) into global memory and a
//      shared copy;
//   5. A22 -= L21 U12 on the FP64 tensor cores (mma.m8n8k4), L21 and U12
//      from shared memory, A22 read and written in global memory.
// Returns the first zero pivot (1-based) or 0; the factorization completes
// either way (LAPACK getrf semantics).
constexpr int LPW = 16;              // panel width
constexpr int LU_LDP = cholb::ld_for(MAXN);  // panel ld (rows of the panel, <= MAXN)
constexpr int LU_LDU = LPW + 4;      // U12 copy, stored U(q, k) at k * LU_LDU + q
constexpr int LU_CHUNK = 64;         // columns per gather / scatter pass of the interchanges

struct LuSmem {
  double P[LU_LDP * LPW];
  double U[MAXN * LU_LDU];
  double stage[2 * LPW * LU_CHUNK];
  double wv[BT / 32];
  int wi[BT / 32];
  int piv[LPW];
  int who[MAXN];
  int src[2 * LPW], dst[2 * LPW];
  int nmove, fail;
};

// C (mt x nt, global, ldc) -= P (mt x kb, shared, ld lds) U (kb x nt, shared,
// U(q, k) at k * ldu + q), kb <= LPW: each warp owns a 16 x 32 part of every
// 64 x 64 block of C (2 x 4 tiles of 8 x 8), accumulators started from C
__device__ void lu_update_dmma(int mt, int nt, int kb, const double *P, int lds, const double *U, int ldu,
                               double *C, long ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
  for (int ib = 0; ib < mt; ib += 64)
    for (int kb0 = 0; kb0 < nt; kb0 += 64) {
      const int r0 = ib + wr, c0 = kb0 + wc;
      if (r0 >= mt || c0 >= nt) continue;  // warp-uniform
      double acc[2][4][2];
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int i = r0 + 8 * a + g, k = c0 + 8 * b + 2 * t + e;
            acc[a][b][e] = (i < mt && k < nt) ? C[i + (long)k * ldc] : 0.0;
          }
#pragma unroll
      for (int q = 0; q < LPW; q += 4) {
        const int qq = q + t;
        double av[2], bv[4];
#pragma unroll
        for (int a = 0; a < 2; a++) {
          const int i = r0 + 8 * a + g;
          av[a] = (i < mt && qq < kb) ? -P[i + qq * lds] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int k = c0 + 8 * b + g;
          bv[b] = (k < nt && qq < kb) ? U[k * ldu + qq] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) cholb::dmma_8x8x4(acc[a][b], av[a], bv[b]);
      }
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int i = r0 + 8 * a + g, k = c0 + 8 * b + 2 * t + e;
            if (i < mt && k < nt) C[i + (long)k * ldc] = acc[a][b][e];
          }
    }
}

// step 1: partial-pivoting LU of the m x jb panel in shared memory; S.piv[c]
// = panel-relative pivot row of column c; returns the first zero pivot
// (1-based, panel-relative) or 0
__device__ int lu_panel(LuSmem &S, int m, int jb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double *P = S.P;
  int fail = 0;
  for (int c = 0; c < jb; c++) {
    double v = -1.0;
    int vi = INT_MAX;
    for (int i = c + tid; i < m; i += BT) {
      const double a = fabs(P[i + c * LU_LDP]);
      if (a > v) { v = a; vi = i; }   // NaN never wins
    }
    for (int o = 16; o; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int oi = __shfl_xor_sync(0xffffffffu, vi, o);
      if (ov > v || (ov == v && oi < vi)) { v = ov; vi = oi; }
    }
    if (lane == 0) { S.wv[warp] = v; S.wi[warp] = vi; }
    __syncthreads();
    double best = -1.0;
    int p = INT_MAX;
    for (int w = 0; w < BT / 32; w++)
      if (S.wv[w] > best || (S.wv[w] == best && S.wi[w] < p)) { best = S.wv[w]; p = S.wi[w]; }
    if (!(best > 0.0)) p = c;  // zero (or NaN) column: no interchange
    if (tid == 0) S.piv[c] = p;
    if (p != c && tid < jb) {
      const double t0 = P[c + tid * LU_LDP];
      P[c + tid * LU_LDP] = P[p + tid * LU_LDP];
      P[p + tid * LU_LDP] = t0;
    }
    __syncthreads();
    const double piv = P[c + c * LU_LDP];
    if (piv == 0.0) {
      if (!fail) fail = c + 1;
    } else {
      const double r = 1.0 / piv;
      const bool use_r = fabs(piv) >= DBL_MIN;
      for (int i = c + 1 + tid; i < m; i += BT) {
        const double l = use_r ? P[i + c * LU_LDP] * r : P[i + c * LU_LDP] / piv;
        P[i + c * LU_LDP] = l;
        for (int k = c + 1; k < jb; k++) P[i + k * LU_LDP] = fma(-l, P[c + k * LU_LDP], P[i + k * LU_LDP]);
      }
    }
    __syncthreads();
  }
  return fail;
}

__device__ int lu_blocked(const Prob &pr, LuSmem &S) {
  const int tid = threadIdx.x, n = pr.n;
  double *A = pr.A;
  const long lda = pr.lda;
  if (tid == 0) S.fail = 0;
  for (int j = 0; j < n; j += LPW) {
    const int jb = min(LPW, n - j), m = n - j, nt = n - j - jb;
    stage_tile(S.P, LU_LDP, A + j + (long)j * lda, lda, m, jb);
    __syncthreads();
    const int f = lu_panel(S, m, jb);
    if (tid == 0 && f && !S.fail) S.fail = j + f;
    for (int idx = tid; idx < m * jb; idx += BT) {
      const int i = idx % m, c = idx / m;
      A[(j + i) + (long)(j + c) * lda] = S.P[i + c * LU_LDP];
    }
    if (tid < jb) pr.ipiv[j + tid] = j + S.piv[tid];
    // the panel's interchanges as one row permutation: who[r] = the panel
    // row whose content ends at row r (panel-relative)
    for (int r = tid; r < m; r += BT) S.who[r] = r;
    __syncthreads();
    if (tid == 0) {
      for (int c = 0; c < jb; c++) {
        const int p = S.piv[c];
        const int t0 = S.who[c];
        S.who[c] = S.who[p];
        S.who[p] = t0;
      }
      int cnt = 0;
      for (int c = 0; c < jb; c++) {  // moved rows: the first jb rows and the pivot rows
        if (S.who[c] != c) { S.dst[cnt] = c; S.src[cnt] = S.who[c]; cnt++; }
        const int p = S.piv[c];
        if (p >= jb && S.who[p] != p) {
          bool seen = false;
          for (int q = 0; q < cnt; q++) seen = seen || S.dst[q] == p;
          if (!seen) { S.dst[cnt] = p; S.src[cnt] = S.who[p]; cnt++; }
        }
      }
      S.nmove = cnt;
    }
    __syncthreads();
    const int nmove = S.nmove;
    if (nmove > 0) {  // gather / scatter over the columns outside the panel, LU_CHUNK at a time
      const int nout = n - jb;
      for (int c0 = 0; c0 < nout; c0 += LU_CHUNK) {
        const int cw = min(LU_CHUNK, nout - c0);
        for (int e = tid; e < nmove * cw; e += BT) {
          const int q = e % nmove, cc = c0 + e / nmove, col = cc < j ? cc : cc + jb;
          S.stage[e] = A[(j + S.src[q]) + (long)col * lda];
        }
        __syncthreads();
        for (int e = tid; e < nmove * cw; e += BT) {
          const int q = e % nmove, cc = c0 + e / nmove, col = cc < j ? cc : cc + jb;
          A[(j + S.dst[q]) + (long)col * lda] = S.stage[e];
        }
        __syncthreads();
      }
    }
    if (nt > 0) {
      // U12 = L11^-1 A12, one thread per column
      for (int k = tid; k < nt; k += BT) {
        double x[LPW];
        double *col = A + j + (long)(j + jb + k) * lda;
#pragma unroll
        for (int q = 0; q < LPW; q++) x[q] = q < jb ? col[q] : 0.0;
#pragma unroll
        for (int q = 0; q < LPW; q++) {
          if (q >= jb) continue;
#pragma unroll
          for (int r = q + 1; r < LPW; r++)
            if (r < jb) x[r] = fma(-S.P[r + q * LU_LDP], x[q], x[r]);
        }
#pragma unroll
        for (int q = 0; q < LPW; q++)
          if (q < jb) {
            col[q] = x[q];
            S.U[k * LU_LDU + q] = x[q];
          }
      }
      __syncthreads();
      if (m > jb) lu_update_dmma(m - jb, nt, jb, S.P + jb, LU_LDP, S.U, LU_LDU, A + (j + jb) + (long)(j + jb) * lda, lda);
      __syncthreads();
    }
  }
  __syncthreads();
  return S.fail;
}

__global__ void __launch_bounds__(BT)
batched_getrf_kernel(const Prob *__restrict__ probs, const int *__restrict__ order, int count,
                     int *__restrict__ next, int *__restrict__ info) {
  extern __shared__ __align__(16) double sm[];
  LuSmem &S = *reinterpret_cast<LuSmem *>(sm);
  __shared__ int s_p;
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) {
      const int t = atomicAdd(next, 1);
      s_p = t < count ? order[t] : -1;
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) return;
    const Prob pr = probs[p];
    const int fail = lu_blocked(pr, S);
    if (tid == 0) info[p] = fail;
    __syncthreads();
  }
}

// P A = L U solves, one right-hand side at a time in shared memory: the
// interchanges in order, then the blocked unit-lower and upper solves
__global__ void __launch_bounds__(BT)
batched_getrs_kernel(const Prob *__restrict__ probs, const int *__restrict__ order, int count,
                     int *__restrict__ next, const int *__restrict__ info) {
  __shared__ int s_p;
  __shared__ double sbv[MAXN];
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) {
      const int t = atomicAdd(next, 1);
      s_p = t < count ? order[t] : -1;
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) return;
    const Prob pr = probs[p];
    if (info[p] == 0) {
      const int n = pr.n;
      for (int r = 0; r < pr.nrhs; r++) {
        double *bg = pr.B + (long)r * pr.ldb;
        for (int i = tid; i < n; i += BT) sbv[i] = bg[i];
        __syncthreads();
        if (tid == 0)
          for (int k = 0; k < n; k++) {
            const int q = pr.ipiv[k];
            if (q != k) { const double t0 = sbv[k]; sbv[k] = sbv[q]; sbv[q] = t0; }
          }
        __syncthreads();
        tri_solve_smem(pr.A, pr.lda, n, sbv, true, true, false);    // L y = P b
        tri_solve_smem(pr.A, pr.lda, n, sbv, false, false, false);  // U x = y
        for (int i = tid; i < n; i += BT) bg[i] = sbv[i];
        __syncthreads();
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host side

struct BatchBufs {
  Prob *probs;
  int *order, *next, *info;
  unsigned char *h, *d;  // pinned staging copy of the problem list, its device copy
  size_t bytes;          // bytes the upload copies
};

// The problem list, sorted by decreasing order, written into the pinned
// staging buffer (host side, every call); enqueue_upload() copies it to the
// device on the stream (a node of the captured graph on replays).
BatchBufs prepare(const std::vector<Prob> &P, int slot_p) {
  const int count = (int)P.size();
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return P[a].n > P[b].n; });
  size_t bytes = sizeof(Prob) * count + sizeof(int) * (2 * count + 64);
  unsigned char *d = (unsigned char *)scratch(slot_p, bytes);
  unsigned char *h = (unsigned char *)pinned(slot_p, bytes);
  memcpy(h, P.data(), sizeof(Prob) * count);
  memcpy(h + sizeof(Prob) * count, order.data(), sizeof(int) * count);
  memset(h + sizeof(Prob) * count + sizeof(int) * count, 0, sizeof(int) * 64);
  BatchBufs b;
  b.probs = (Prob *)d;
  b.order = (int *)(d + sizeof(Prob) * count);
  b.next = b.order + count;
  b.info = b.next + 64;
  b.h = h;
  b.d = d;
  b.bytes = bytes - sizeof(int) * count;
  return b;
}

void enqueue_upload(const BatchBufs &b, cudaStream_t st) {
  ATLB_CUDA_CHECK(cudaMemcpyAsync(b.d, b.h, b.bytes, cudaMemcpyHostToDevice, st));
}

int grid_size(size_t smem) {
  int per_sm = smem > 100 * 1024 ? 1 : (smem > 60 * 1024 ? 2 : 4);
  return num_sms() * per_sm;
}

}  // namespace

// One batched Cholesky + solve: upload, one persistent launch, info back to
// info_out (pinned).  The launch sequence depends only on the batch's shape
// and the buffers, so it is replayed from a CUDA graph from the third call on
// (run_graph): the problem list itself travels in the captured copy.
void batched_posv_dev(const std::vector<Prob> &P, int *info_out, cudaStream_t st) {
  const int count = (int)P.size();
  if (!count) return;
  BatchBufs b = prepare(P, kSlotBatch0);
  int maxn = 0;
  for (auto &p : P) maxn = std::max(maxn, p.n);
  const int SMALL = tune(kTuneBatchPosvSmall), PW = tune(kTuneBatchPosvPW);
  const int sn = std::min(maxn, SMALL);
  const size_t sm_bytes = std::max(sizeof(double) * sn * cholb::ld_for(sn),
                                   maxn > SMALL ? sizeof(double) * (size_t)cholb::ld_for(maxn) * PW : (size_t)0);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(batched_posv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    configured = true;
  }
  const std::vector<unsigned long long> key = {0xBA7C0001ull, (unsigned long long)tune_generation(),
      (unsigned long long)count, (unsigned long long)maxn, (unsigned long long)(uintptr_t)b.d,
      (unsigned long long)(uintptr_t)b.h, (unsigned long long)(uintptr_t)info_out,
      (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    enqueue_upload(b, st);
    batched_posv_kernel<<<grid_size(sm_bytes), BT, sm_bytes, st>>>(b.probs, b.order, count, b.next, b.info, SMALL,
                                                                    PW);
    ATLB_CUDA_CHECK(cudaGetLastError());
    ATLB_CUDA_CHECK(cudaMemcpyAsync(info_out, b.info, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
  });
}

// Batched LU (+ the solve when nrhs > 0 for the problems), the same way.
void batched_gesv_dev(const std::vector<Prob> &P, bool solve, int *info_out, cudaStream_t st) {
  const int count = (int)P.size();
  if (!count) return;
  BatchBufs b = prepare(P, kSlotBatch0);
  int maxn = 0;
  for (auto &p : P) maxn = std::max(maxn, p.n);
  const size_t smb = sizeof(LuSmem);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(batched_getrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb));
    configured = true;
  }
  const std::vector<unsigned long long> key = {0xBA7C0002ull + (solve ? 1 : 0),
      (unsigned long long)tune_generation(), (unsigned long long)count, (unsigned long long)maxn,
      (unsigned long long)(uintptr_t)b.d, (unsigned long long)(uintptr_t)b.h,
      (unsigned long long)(uintptr_t)info_out, (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    enqueue_upload(b, st);
    batched_getrf_kernel<<<grid_size(smb), BT, smb, st>>>(b.probs, b.order, count, b.next, b.info);
    ATLB_CUDA_CHECK(cudaGetLastError());
    if (solve) {
      ATLB_CUDA_CHECK(cudaMemsetAsync(b.next, 0, sizeof(int), st));
      batched_getrs_kernel<<<num_sms() * 4, BT, 0, st>>>(b.probs, b.order, count, b.next, b.info);
      ATLB_CUDA_CHECK(cudaGetLastError());
    }
    ATLB_CUDA_CHECK(cudaMemcpyAsync(info_out, b.info, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
  });
}

}  // namespace atlb

using namespace atlb;

extern "C" {

// Batched Cholesky factor + solve of `count` independent SPD systems (lower
// triangle referenced, column-major): A[i] (n[i] x n[i], lda[i]) and B[i]
// (n[i] x nrhs[i], ldb[i]) are DEVICE pointers; on return A[i] holds L and
// B[i] the solution, info[i] (host array) the potrf info.  One persistent
// launch; orders up to 256.  Returns 0 or a negative argument position.
int atlb_dposv_batched(int count, const int *n, double *const *A, const int *lda, double *const *B,
                       const int *ldb, const int *nrhs, int *info) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  std::vector<Prob> P(count);
  for (int i = 0; i < count; i++) {
    if (n[i] < 0 || n[i] > MAXN) return -2;
    if (lda[i] < std::max(1, n[i])) return -4;
    if (ldb[i] < std::max(1, n[i])) return -6;
    if (nrhs[i] < 0) return -7;
    P[i] = {A[i], B[i], nullptr, n[i], lda[i], ldb[i], nrhs[i]};
  }
  cudaStream_t st = stream();
  int *hinfo = (int *)pinned(kSlotBatch1, sizeof(int) * count);
  batched_posv_dev(P, hinfo, st);
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  memcpy(info, hinfo, sizeof(int) * count);
  return 0;
}

// Batched LU with partial pivoting (+ optional solve when B is non-NULL):
// device pointers as above; ipiv[i] device int arrays of n[i] entries
// (0-based), info[i] host.  Orders up to 256.
int atlb_dgesv_batched(int count, const int *n, double *const *A, const int *lda, int *const *ipiv,
                       double *const *B, const int *ldb, const int *nrhs, int *info) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  std::vector<Prob> P(count);
  for (int i = 0; i < count; i++) {
    if (n[i] < 0 || n[i] > MAXN) return -2;
    if (lda[i] < std::max(1, n[i])) return -4;
    if (B && (ldb[i] < std::max(1, n[i]) || nrhs[i] < 0)) return -7;
    P[i] = {A[i], B ? B[i] : nullptr, ipiv[i], n[i], lda[i], B ? ldb[i] : 1, B ? nrhs[i] : 0};
  }
  cudaStream_t st = stream();
  int *hinfo = (int *)pinned(kSlotBatch1, sizeof(int) * count);
  batched_gesv_dev(P, B != nullptr, hinfo, st);
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  memcpy(info, hinfo, sizeof(int) * count);
  return 0;
}

// Batched LU with partial pivoting only (LAPACK getrf semantics per problem:
// A[i] overwritten by L\U, ipiv[i] 0-based device arrays, info[i] host).
int atlb_dgetrf_batched(int count, const int *n, double *const *A, const int *lda, int *const *ipiv, int *info) {
  return atlb_dgesv_batched(count, n, A, lda, ipiv, nullptr, nullptr, nullptr, info);
}

}  // extern "C"
