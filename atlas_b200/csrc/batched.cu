// Batched factorizations and solves of many small, uneven-size systems.  No
// counterpart in the reference (ATLAS factors one matrix per call); the
// per-problem arithmetic is that of ATL_potrfL / ATL_getf2 / ATL_potrs /
// ATL_getrs on a single small matrix.
//
// One persistent launch per batch: CTAs pull problem indices from an atomic
// counter over a work list sorted by decreasing size (largest first, so the
// tail of the launch is made of small problems), and each problem is handled
// entirely by one CTA.  Size buckets pick the code path: a matrix of order
// <= 96 is factored with the whole matrix in shared memory; larger ones
// (up to 256) in 32-column panels staged in shared memory with the trailing
// update written back to global memory (L2-resident at these sizes).
// Nothing waits on another CTA, so the launch cannot stall.
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
// Size buckets (tunable, tuning.cu): orders up to batch_posv_small (Cholesky)
// / batch_getrf_smem (LU) are factored whole in shared memory, larger ones in
// panels of batch_posv_pw columns.

struct Prob {
  double *A;
  double *B;
  int *ipiv;
  int n, lda, ldb, nrhs;
};

// ---------------------------------------------------------------- Cholesky

// forward then backward substitution with L (lower, in shared memory or
// global, ld = ldl) for nrhs columns of B (global)
__device__ void chol_solve(const double *L, int ldl, int n, double *B, int ldb, int nrhs) {
  const int tid = threadIdx.x;
  for (int r = 0; r < nrhs; r++) {
    double *b = B + (long)r * ldb;
    for (int j = 0; j < n; j++) {  // L y = b
      const double yj = b[j] / L[j + (long)j * ldl];
      __syncthreads();
      if (tid == 0) b[j] = yj;
      for (int i = j + 1 + tid; i < n; i += BT) b[i] = fma(-L[i + (long)j * ldl], yj, b[i]);
      __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {  // L^T x = y
      const double xj = b[j] / L[j + (long)j * ldl];
      __syncthreads();
      if (tid == 0) b[j] = xj;
      for (int i = tid; i < j; i += BT) b[i] = fma(-L[j + (long)i * ldl], xj, b[i]);
      __syncthreads();
    }
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
      for (int idx = tid; idx < n * n; idx += BT) sm[idx % n + (idx / n) * lds] = pr.A[idx % n + (long)(idx / n) * pr.lda];
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
        for (int idx = tid; idx < m * jb; idx += BT)
          sm[idx % m + (idx / m) * lds] = pr.A[j + idx % m + (long)(j + idx / m) * pr.lda];
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

// partial-pivoting LU of the n x n matrix in shared memory (ld lds); ipiv
// 0-based; returns the first zero pivot (1-based) or 0.  Pivot rule as
// ATL_getf2: first maximal |a| (ties to the lowest row index).
__device__ int lu_smem(double *s, int lds, int n, int *ipiv, double *wv, int *wi) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int fail = 0;
  for (int j = 0; j < n; j++) {
    double v = -1.0;
    int vi = INT_MAX;
    for (int i = j + tid; i < n; i += BT) {
      const double t = fabs(s[i + j * lds]);
      if (t > v) { v = t; vi = i; }
    }
    for (int o = 16; o; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, v, o);
      const int oi = __shfl_xor_sync(0xffffffffu, vi, o);
      if (ov > v || (ov == v && oi < vi)) { v = ov; vi = oi; }
    }
    if (lane == 0) { wv[warp] = v; wi[warp] = vi; }
    __syncthreads();
    double best = -1.0;
    int p = INT_MAX;
    for (int w = 0; w < BT / 32; w++)
      if (wv[w] > best || (wv[w] == best && wi[w] < p)) { best = wv[w]; p = wi[w]; }
    if (best <= 0.0) p = j;
    if (tid == 0) ipiv[j] = p;
    if (p != j)
      for (int c = tid; c < n; c += BT) {
        const double t = s[j + c * lds];
        s[j + c * lds] = s[p + c * lds];
        s[p + c * lds] = t;
      }
    __syncthreads();
    const double piv = s[j + j * lds];
    if (piv == 0.0) {
      if (!fail) fail = j + 1;
    } else {
      const double r = 1.0 / piv;
      const bool use_r = fabs(piv) >= DBL_MIN;
      for (int i = j + 1 + tid; i < n; i += BT) s[i + j * lds] = use_r ? s[i + j * lds] * r : s[i + j * lds] / piv;
      __syncthreads();
      // rank-1 update: 16 x 16 threads, rows tx + 16 a, columns ty + 16 b
      const int tx = tid % 16, ty = tid / 16;
      for (int k = j + 1 + ty; k < n; k += 16) {
        const double u = s[j + k * lds];
        for (int i = j + 1 + tx; i < n; i += 16) s[i + k * lds] = fma(-s[i + j * lds], u, s[i + k * lds]);
      }
    }
    __syncthreads();
  }
  return fail;
}

__global__ void __launch_bounds__(BT)
batched_getrf_kernel(const Prob *__restrict__ probs, const int *__restrict__ order, int count,
                     int *__restrict__ next, int sm_max, int *__restrict__ info) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_p;
  __shared__ double wv[BT / 32];
  __shared__ int wi[BT / 32];
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
    int fail;
    if (n <= sm_max) {  // the whole matrix in shared memory
      const int lds = n + 1;
      for (int idx = tid; idx < n * n; idx += BT) sm[idx % n + (idx / n) * lds] = pr.A[idx % n + (long)(idx / n) * pr.lda];
      __syncthreads();
      fail = lu_smem(sm, lds, n, pr.ipiv, wv, wi);
      for (int idx = tid; idx < n * n; idx += BT) pr.A[idx % n + (long)(idx / n) * pr.lda] = sm[idx % n + (idx / n) * lds];
    } else {  // in place in global memory (L2-resident at these orders)
      fail = lu_smem(pr.A, pr.lda, n, pr.ipiv, wv, wi);
    }
    if (tid == 0) info[p] = fail;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(BT)
batched_getrs_kernel(const Prob *__restrict__ probs, const int *__restrict__ order, int count,
                     int *__restrict__ next, const int *__restrict__ info) {
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
    if (info[p] == 0) {
      const int n = pr.n;
      const int *ipiv = pr.ipiv;
      const double *L = pr.A;
      for (int r = 0; r < pr.nrhs; r++) {
        double *b = pr.B + (long)r * pr.ldb;
        if (tid == 0)
          for (int k = 0; k < n; k++) {
            const int q = ipiv[k];
            if (q != k) { const double t = b[k]; b[k] = b[q]; b[q] = t; }
          }
        __syncthreads();
        for (int j = 0; j < n; j++) {  // unit lower
          const double yj = b[j];
          __syncthreads();
          for (int i = j + 1 + tid; i < n; i += BT) b[i] = fma(-L[i + (long)j * pr.lda], yj, b[i]);
          __syncthreads();
        }
        for (int j = n - 1; j >= 0; j--) {  // upper
          const double xj = b[j] / L[j + (long)j * pr.lda];
          __syncthreads();
          if (tid == 0) b[j] = xj;
          for (int i = tid; i < j; i += BT) b[i] = fma(-L[i + (long)j * pr.lda], xj, b[i]);
          __syncthreads();
        }
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
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(batched_getrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    configured = true;
  }
  const int sm_max = std::min(maxn, tune(kTuneBatchGetrfSmem));  // FP64 in shared memory: 206 KB at 160
  const size_t smb = sizeof(double) * (size_t)sm_max * (sm_max + 1);
  const std::vector<unsigned long long> key = {0xBA7C0002ull + (solve ? 1 : 0),
      (unsigned long long)tune_generation(), (unsigned long long)count, (unsigned long long)maxn,
      (unsigned long long)(uintptr_t)b.d, (unsigned long long)(uintptr_t)b.h,
      (unsigned long long)(uintptr_t)info_out, (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    enqueue_upload(b, st);
    batched_getrf_kernel<<<grid_size(smb), BT, smb, st>>>(b.probs, b.order, count, b.next, sm_max, b.info);
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
