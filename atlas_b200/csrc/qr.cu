// Householder QR (clapack_dgeqrf / ATL_dgeqrf), ATLAS conventions: reflector
// H = I - tau v v^T with v(0) = 1, beta = -sign(alpha)*||(alpha, x)|| (sign(0)
// = +), tau = (beta - alpha)/beta, v = x/(alpha - beta), R(j,j) = beta
// (src/lapack/ATL_larfg.c:120-189).
//
// Driver: the reference's blocked loop (src/lapack/ATL_geqrf.c:145-191):
// panels of NBQ columns, each factored and its block reflector I - V T V^T
// applied to the columns on its right (ATL_larfb Left/Trans/Forward/Columnwise,
// src/lapack/ATL_larfb.c:156-240).  Inside a panel, leaves of <= 32 columns
// are factored by one cluster kernel (ATL_geqr2's column loop,
// src/lapack/ATL_geqr2.c:100-142) and applied to the rest of the panel, as
// the reference's recursive panel ATL_geqrr does.  V is copied out with its
// implicit unit diagonal and zeros made explicit, so every block-reflector
// product is a plain DMMA GEMM; T is built from the Gram matrix V^T V
// (ATL_larft's recurrence, src/lapack/ATL_larft.c:646).
//
// Panel kernel: the panel's rows live in registers across a cluster of up to
// 16 CTAs.  Column j needs a single cluster-wide reduction: the dot products
// s_k = sum_{i>j} a_ij a_ik for k >= j (s_j = ||x||^2) give beta, tau and
// w = v^T A in closed form (w_k = a_jk + s_k/(alpha-beta)).
#include <algorithm>
#include <cooperative_groups.h>
#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace atlb {
namespace {

constexpr int QT = 512;
constexpr int NBQ_MAX = 128;  // largest outer panel width (the trailing update's K)

template <int NB>
struct QPub {
  double s[NB];    // this CTA's partial dot products
  double row[NB];  // row j (published by its owner, CTA 0)
};

// lane l returns sum over the warp of v[l % NB]; v is destroyed
template <int NB>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[NB], int lane) {
#pragma unroll
  for (int s = NB / 2; s >= 1; s >>= 1) {
    const bool upper = lane & s;
#pragma unroll
    for (int i = 0; i < s; i++) {
      double send = upper ? v[i] : v[i + s];
      double keep = upper ? v[i + s] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  double r = v[0];
#pragma unroll
  for (int o = NB; o < 32; o <<= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  return r;
}

template <int NB, int RPT>
__global__ void __launch_bounds__(QT, 1)
geqr2_cluster_kernel(int M, int ncols, double *__restrict__ A, long lda, double *__restrict__ tau) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), crank = (int)cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int TOT = C * QT;
  const int K = min(M, ncols);

  __shared__ QPub<NB> pub[2];
  __shared__ double red[QT / 32][NB];
  __shared__ double ssum[NB];
  __shared__ double srow[NB];

  double a[RPT][NB];
  int rows[RPT];
#pragma unroll
  for (int q = 0; q < RPT; q++) {
    int r = crank * QT + tid + q * TOT;
    rows[q] = r;
#pragma unroll
    for (int k = 0; k < NB; k++) a[q][k] = (r < M && k < ncols) ? A[r + (long)k * lda] : 0.0;
  }

#pragma unroll
  for (int j = 0; j < NB; j++) {
    if (j >= K) break;
    const int b = j & 1;
    // partial dot products of column j with columns j.. over my rows below j
    double p[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) p[k] = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
      if (rows[q] > j && rows[q] < M) {
#pragma unroll
        for (int k = j; k < NB; k++) p[k] = fma(a[q][j], a[q][k], p[k]);
      }
      if (rows[q] == j) {
#pragma unroll
        for (int k = 0; k < NB; k++) pub[b].row[k] = a[q][k];
      }
    }
    double ws = warp_reduce_scatter<NB>(p, lane);
    if (lane < NB) red[warp][lane] = ws;
    __syncthreads();
    if (tid < NB) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < QT / 32; w++) t += red[w][tid];
      pub[b].s[tid] = t;
    }
    cl.sync();
    // gather every CTA's partial sums and row j
    if (tid < NB) {
      double t = 0.0;
      for (int r = 0; r < C; r++) t += cl.map_shared_rank(&pub[b], r)->s[tid];
      ssum[tid] = t;
      srow[tid] = cl.map_shared_rank(&pub[b], 0)->row[tid];
    }
    __syncthreads();
    const double alpha = srow[j], xn2 = ssum[j];
    double t_ = 0.0, beta = alpha, scale = 0.0;
    if (xn2 != 0.0) {
      const double bp = sqrt(fma(alpha, alpha, xn2));
      beta = alpha >= 0.0 ? -bp : bp;
      t_ = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    if (crank == 0 && tid == 0) tau[j] = t_;
    if (t_ != 0.0) {
#pragma unroll
      for (int q = 0; q < RPT; q++) {
        if (rows[q] > j && rows[q] < M) {
          const double v = a[q][j] * scale;
          a[q][j] = v;
          const double tv = t_ * v;
#pragma unroll
          for (int k = j + 1; k < NB; k++) a[q][k] = fma(-tv, fma(scale, ssum[k], srow[k]), a[q][k]);
        } else if (rows[q] == j) {
          a[q][j] = beta;
#pragma unroll
          for (int k = j + 1; k < NB; k++) a[q][k] = fma(-t_, fma(scale, ssum[k], srow[k]), a[q][k]);
        }
      }
    }
    // ssum/srow/red are rewritten next column only after two more barriers
  }
#pragma unroll
  for (int q = 0; q < RPT; q++) {
    if (rows[q] < M) {
#pragma unroll
      for (int k = 0; k < NB; k++)
        if (k < ncols) A[rows[q] + (long)k * lda] = a[q][k];
    }
  }
  cl.sync();
}

// Fallback for panels taller than a cluster holds: one CTA in global memory.
__global__ void __launch_bounds__(1024)
geqr2_global_kernel(int M, int ncols, double *A, long lda, double *tau) {
  __shared__ double red[32];
  __shared__ double w[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x / 32;
  const int K = min(M, ncols);
  for (int j = 0; j < K; j++) {
    double *cj = A + (long)j * lda;
    double s = 0.0;
    for (int i = j + 1 + tid; i < M; i += blockDim.x) s += cj[i] * cj[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    double xn2 = 0.0;
    for (int q = 0; q < nw; q++) xn2 += red[q];
    const double alpha = cj[j];
    double t_ = 0.0, beta = alpha, scale = 0.0;
    if (xn2 != 0.0) {
      const double bp = sqrt(fma(alpha, alpha, xn2));
      beta = alpha >= 0.0 ? -bp : bp;
      t_ = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    __syncthreads();
    if (tid == 0) tau[j] = t_;
    if (t_ != 0.0) {
      for (int i = j + 1 + tid; i < M; i += blockDim.x) cj[i] *= scale;
      __syncthreads();
      if (tid == 0) cj[j] = 1.0;
      __syncthreads();
      for (int k = j + 1; k < ncols; k++) {
        double *ck = A + (long)k * lda;
        double d = 0.0;
        for (int i = j + tid; i < M; i += blockDim.x) d += cj[i] * ck[i];
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) red[warp] = d;
        __syncthreads();
        if (tid == 0) {
          double t = 0.0;
          for (int q = 0; q < nw; q++) t += red[q];
          w[0] = t * t_;
        }
        __syncthreads();
        const double wk = w[0];
        for (int i = j + tid; i < M; i += blockDim.x) ck[i] -= cj[i] * wk;
        __syncthreads();
      }
      if (tid == 0) cj[j] = beta;
    }
    __syncthreads();
  }
}

int g_qr_max_cluster = 0;

template <int NB, int RPT>
void launch_geqr2_cluster(int M, int ncols, double *A, long lda, double *tau, cudaStream_t st) {
  int C = cdiv(M, QT * RPT);
  auto kern = geqr2_cluster_kernel<NB, RPT>;
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    configured = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(QT, 1, 1);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATLB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, M, ncols, A, lda, tau));
}

void init_qr_cluster() {
  if (g_qr_max_cluster) return;
  auto kern = geqr2_cluster_kernel<32, 1>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16, 1, 1);
  cfg.blockDim = dim3(QT, 1, 1);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) { cudaGetLastError(); n = 0; }
  g_qr_max_cluster = n > 0 ? 16 : 8;
}

// leaf width supported for M rows
int qr_leaf(int M) {
  init_qr_cluster();
  if (M <= g_qr_max_cluster * QT) return 32;
  if (M <= g_qr_max_cluster * QT * 2) return 16;
  return 8;
}

void geqr2_leaf(int M, int ncols, double *A, long lda, double *tau, cudaStream_t st) {
  if (ncols <= 32 && M <= g_qr_max_cluster * QT) launch_geqr2_cluster<32, 1>(M, ncols, A, lda, tau, st);
  else if (ncols <= 16 && M <= g_qr_max_cluster * QT * 2) launch_geqr2_cluster<16, 2>(M, ncols, A, lda, tau, st);
  else if (ncols <= 8 && M <= g_qr_max_cluster * QT * 4) launch_geqr2_cluster<8, 4>(M, ncols, A, lda, tau, st);
  else {
    geqr2_global_kernel<<<1, 1024, 0, st>>>(M, ncols, A, lda, tau);
    ATLB_CUDA_CHECK(cudaGetLastError());
  }
}

// V (M x k, ld M) = unit lower trapezoid of the factored panel at P
__global__ void extract_v_kernel(int M, int k, const double *P, long ldp, double *V) {
  long total = (long)M * k;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    V[idx] = (i > j) ? P[i + (long)j * ldp] : (i == j ? 1.0 : 0.0);
  }
}

// T (k x k upper, ld k) from G = V^T V and tau: T(0:i,i) = -tau_i T(0:i,0:i) G(0:i,i)
__global__ void __launch_bounds__(256) larft_kernel(int k, const double *G, const double *tau, double *T) {
  extern __shared__ double sT[];  // k x k
  const int tid = threadIdx.x;
  for (int idx = tid; idx < k * k; idx += blockDim.x) sT[idx] = 0.0;
  __syncthreads();
  for (int i = 0; i < k; i++) {
    const double ti = tau[i];
    double val = 0.0;
    if (tid < i) {
      for (int q = tid; q < i; q++) val += sT[tid + q * k] * G[q + (long)i * k];
      val *= -ti;
    }
    __syncthreads();
    if (tid < i) sT[tid + i * k] = val;
    if (tid == 0) sT[i + i * k] = ti;
    __syncthreads();
  }
  for (int idx = tid; idx < k * k; idx += blockDim.x) T[idx] = sT[idx];
}

// C (m x n, ldc) = (I - V T V^T)^T C, V explicit (m x k, ld m), T k x k
void larfb_lt(int m, int n, int k, const double *V, const double *T, double *C, long ldc,
              double *W, cudaStream_t st) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  double *W1 = W, *W2 = W + (size_t)k * n;
  dgemm_dev(kTrans, kNoTrans, k, n, m, 1.0, V, m, C, ldc, 0.0, W1, k, st);
  dgemm_dev(kTrans, kNoTrans, k, n, k, 1.0, T, k, W1, k, 0.0, W2, k, st);
  dgemm_dev(kNoTrans, kNoTrans, m, n, k, -1.0, V, m, W2, k, 1.0, C, ldc, st);
}

void build_vt(int m, int k, const double *P, long ldp, const double *tau, double *V, double *G,
              double *T, cudaStream_t st) {
  long tot = (long)m * k;
  extract_v_kernel<<<(int)std::min<long>((tot + 255) / 256, 8192), 256, 0, st>>>(m, k, P, ldp, V);
  ATLB_CUDA_CHECK(cudaGetLastError());
  dgemm_dev(kTrans, kNoTrans, k, k, m, 1.0, V, m, V, m, 0.0, G, k, st);
  size_t sm = sizeof(double) * k * k;
  static bool cfg = false;
  if (!cfg) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(double) * NBQ_MAX * NBQ_MAX)));
    cfg = true;
  }
  larft_kernel<<<1, 256, sm, st>>>(k, G, tau, T);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// Apply the block reflector H = I - V T V^T (V explicit, len x k) or its
// transpose to C: from the left (C is len x n) or the right (C is m x len).
void larfb_gen(int side, int trans, int len, int other, int k, const double *V, const double *T, double *C,
               long ldc, double *W, cudaStream_t st) {
  if (len <= 0 || other <= 0 || k <= 0) return;
  const int tt = trans == kNoTrans ? kNoTrans : kTrans;  // H^T = I - V T^T V^T
  if (side == kLeft) {  // C (len x other) -= V op(T) V^T C
    double *W1 = W, *W2 = W + (size_t)k * other;
    dgemm_dev(kTrans, kNoTrans, k, other, len, 1.0, V, len, C, ldc, 0.0, W1, k, st);
    dgemm_dev(tt, kNoTrans, k, other, k, 1.0, T, k, W1, k, 0.0, W2, k, st);
    dgemm_dev(kNoTrans, kNoTrans, len, other, k, -1.0, V, len, W2, k, 1.0, C, ldc, st);
  } else {              // C (other x len) -= C V op(T) V^T
    double *W1 = W, *W2 = W + (size_t)other * k;
    dgemm_dev(kNoTrans, kNoTrans, other, k, len, 1.0, C, ldc, V, len, 0.0, W1, other, st);
    dgemm_dev(kNoTrans, tt, other, k, k, 1.0, W1, other, T, k, 0.0, W2, other, st);
    dgemm_dev(kNoTrans, kTrans, other, len, k, -1.0, W2, other, V, len, 1.0, C, ldc, st);
  }
}

}  // namespace

// Q = H(0) H(1) ... H(K-1) from dgeqrf_dev's reflectors (columns of A below
// the diagonal, tau) applied to C (M x N): Q C, Q^T C (Left; Q of order M) or
// C Q, C Q^T (Right; Q of order N).  ATL_ormqr's operation
// (src/lapack/ATL_ormqr.c:24), blocked: NBQ reflectors at a time as one block
// reflector I - V T V^T (T from the Gram matrix V^T V, as in the
// factorization), applied with three GEMMs.
void dormqr_dev(int side, int trans, int M, int N, int K, const double *A, long lda, const double *tau,
                double *C, long ldc, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return;
  const int NBQ = tune(kTuneQrNB);
  const int nq = side == kLeft ? M : N;   // order of Q
  const int other = side == kLeft ? N : M;
  size_t need = (size_t)nq * NBQ + 2 * (size_t)NBQ * NBQ + 2 * (size_t)NBQ * other;
  double *ws = (double *)scratch(kSlotQrApply, sizeof(double) * need);
  double *V = ws, *G = V + (size_t)nq * NBQ, *T = G + (size_t)NBQ * NBQ, *W = T + (size_t)NBQ * NBQ;
  const int nblk = cdiv(K, NBQ);
  // Q C = H0 (H1 (... C)): last block first; Q^T C: first block first (Left).
  // C Q = ((C H0) H1) ...: first block first; C Q^T: last block first (Right).
  const bool forward = (side == kLeft) == (trans != kNoTrans);
  for (int t = 0; t < nblk; t++) {
    const int b = forward ? t : nblk - 1 - t;
    const int j = b * NBQ, kb = std::min(NBQ, K - j), len = nq - j;
    build_vt(len, kb, A + j + (long)j * lda, lda, tau + j, V, G, T, st);
    if (side == kLeft) larfb_gen(kLeft, trans, len, other, kb, V, T, C + j, ldc, W, st);
    else larfb_gen(kRight, trans, len, other, kb, V, T, C + (long)j * ldc, ldc, W, st);
  }
}

void dgeqrf_dev(int M, int N, double *A, long lda, double *tau, cudaStream_t st) {
  const int mn = std::min(M, N);
  if (mn <= 0) return;
  const int NBQ = tune(kTuneQrNB);  // the outer panel width (ATL_ilaenv's NB, tuned)
  // workspace: V (M x NBQ), G and T (NBQ x NBQ each), W (2 x NBQ x N)
  size_t need = (size_t)M * NBQ + 2 * (size_t)NBQ * NBQ + 2 * (size_t)NBQ * N;
  double *ws = (double *)scratch(kSlotWork, sizeof(double) * need);
  double *V = ws, *G = V + (size_t)M * NBQ, *T = G + (size_t)NBQ * NBQ, *W = T + (size_t)NBQ * NBQ;
  for (int j = 0; j < mn; j += NBQ) {
    const int nb = std::min(NBQ, mn - j), m = M - j;
    double *P = A + j + (long)j * lda;
    // factor the panel in leaves, applying each leaf to the panel's remaining columns
    for (int l = 0; l < nb;) {
      const int leaf = std::min(qr_leaf(m - l), nb - l);
      double *L = P + l + (long)l * lda;
      geqr2_leaf(m - l, leaf, L, lda, tau + j + l, st);
      if (l + leaf < nb) {
        build_vt(m - l, leaf, L, lda, tau + j + l, V, G, T, st);
        larfb_lt(m - l, nb - l - leaf, leaf, V, T, L + (long)leaf * lda, lda, W, st);
      }
      l += leaf;
    }
    if (j + nb < N) {
      build_vt(m, nb, P, lda, tau + j, V, G, T, st);
      larfb_lt(m, N - j - nb, nb, V, T, P + (long)nb * lda, lda, W, st);
    }
  }
}

}  // namespace atlb
