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
constexpr int NBQ_MAX = 128;  // widest panel factored in one piece (wider panels: two halves)

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

// T (k x k upper, ld ldt, k <= NBQ_MAX) of the block reflector
// H(0) H(1) ... H(k-1) = I - V T V^T, from G = V^T V and tau.  ATL_larft's
// column recurrence T(0:i,i) = -tau_i T(0:i,0:i) G(0:i,i), T(i,i) = tau_i
// runs on the 16-column diagonal blocks (one warp each, all at once); the
// blocks are then merged pairwise, 16 -> 32 -> 64 -> 128, with the identity
// H1 H2 = I - [V1 V2] [T1, -T1 (V1^T V2) T2; 0, T2] [V1 V2]^T, i.e.
// T12 = -T1 G12 T2 (two small products in shared memory per level).
// G's strictly upper part is overwritten in place by T's.
constexpr int LFT_LD = NBQ_MAX + 1;
__global__ void __launch_bounds__(256) larft_kernel(int k, const double *G, long ldg, const double *tau, double *T,
                                                    long ldt) {
  extern __shared__ double lft_smem[];
  double *S = lft_smem;                      // k x k, ld LFT_LD: G, then T
  double *W = lft_smem + NBQ_MAX * LFT_LD;   // products G12 T2 of one level (<= NBQ_MAX^2 / 4 doubles)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int base = 0; base < k * k; base += 256 * 8) {  // eight loads in flight per thread
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, r = idx % k, c = idx / k;
      v[u] = (idx < k * k && r < c) ? G[r + (long)c * ldg] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid;
      if (idx < k * k) S[idx % k + (idx / k) * LFT_LD] = v[u];
    }
  }
  __syncthreads();
  for (int b = warp; b * 16 < k; b += 8) {   // diagonal blocks by the recurrence
    const int o = b * 16, kb = min(16, k - o);
    double *B = S + o + o * LFT_LD;
    for (int i = 0; i < kb; i++) {
      double val = 0.0;
      if (lane < i) {
        for (int q = lane; q < i; q++) val = fma(B[lane + q * LFT_LD], B[q + i * LFT_LD], val);
        val *= -tau[o + i];
      }
      __syncwarp();  // column i of G read by every lane before it is overwritten
      if (lane < i) B[lane + i * LFT_LD] = val;
      if (lane == i) B[i + i * LFT_LD] = tau[o + i];
      __syncwarp();
    }
  }
  __syncthreads();
  for (int h = 16; h < k; h *= 2) {          // merge sibling blocks of order h
    const int npair = (k + 2 * h - 1) / (2 * h);
    // W_p = G12 T2 (h x h2): G12 = S[o : o+h, o+h : o+h+h2], T2 upper h2 x h2
    for (int idx = tid; idx < npair * h * h; idx += 256) {
      const int p = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h;
      const int o = 2 * h * p, h2 = min(h, k - o - h);
      if (h2 <= 0 || c >= h2) continue;
      const double *G12 = S + o + (o + h) * LFT_LD, *T2 = S + (o + h) + (o + h) * LFT_LD;
      double v = 0.0;
      for (int q = 0; q <= c; q++) v = fma(G12[r + q * LFT_LD], T2[q + c * LFT_LD], v);
      W[p * h * h + r + c * h] = v;
    }
    __syncthreads();
    // T12 = -T1 W_p, T1 upper h x h
    for (int idx = tid; idx < npair * h * h; idx += 256) {
      const int p = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h;
      const int o = 2 * h * p, h2 = min(h, k - o - h);
      if (h2 <= 0 || c >= h2) continue;
      const double *T1 = S + o + o * LFT_LD;
      const double *Wp = W + p * h * h;
      double v = 0.0;
      for (int q = r; q < h; q++) v = fma(T1[r + q * LFT_LD], Wp[q + c * h], v);
      S[(o + r) + (o + h + c) * LFT_LD] = -v;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < k * k; idx += 256) {
    const int r = idx % k, c = idx / k;
    T[r + (long)c * ldt] = r <= c ? S[r + c * LFT_LD] : 0.0;
  }
}

constexpr size_t larft_smem_bytes() { return sizeof(double) * ((size_t)NBQ_MAX * LFT_LD + NBQ_MAX * NBQ_MAX / 4); }

// ---- Applying a leaf's reflectors to the rest of its panel.  The leaf is
// m x kb (kb <= 32) with V its unit lower trapezoid, C the n2 panel columns
// on its right (kb + n2 <= NBQ_MAX).  C <- (I - V T V^T)^T C as three
// streaming passes over the rows, in place of GEMMs whose output (kb x n2)
// is too small to fill the GPU:
//   1. qr_leaf_gram_kernel: per-CTA partial sums of V^T [V C] (kb x (kb+n2));
//   2. qr_leaf_reduce_kernel: the partials summed in a fixed order;
//   3. qr_leaf_apply_kernel: every CTA forms T from G = V^T V (the column
//      recurrence) and Y = T^T (V^T C), then C -= V Y for its rows.
// V is read straight from the factored leaf (unit diagonal and zeros above
// it applied on the fly).
constexpr int QL_GRID = 256;         // CTAs of the partial-sum pass (at most)
constexpr int QL_OUT = 32 * NBQ_MAX; // doubles per partial (kb <= 32 rows of <= NBQ_MAX columns)

__device__ __forceinline__ double leaf_v(const double *L, long lda, int r, int a) {
  return r > a ? L[r + (long)a * lda] : (r == a ? 1.0 : 0.0);
}

template <int KB>
__global__ void __launch_bounds__(256) qr_leaf_gram_kernel(int m, int kb, int ncol, const double *L, long lda,
                                                           int rpc, double *part) {
  __shared__ double X[NBQ_MAX][33];  // 32 rows of [V C], column by column
  constexpr int SB = 256 / KB, NJ = NBQ_MAX / SB;
  const int tid = threadIdx.x, a = tid % KB, b0 = tid / KB;
  double acc[NJ];
#pragma unroll
  for (int j = 0; j < NJ; j++) acc[j] = 0.0;
  const int rb = blockIdx.x * rpc, re = min(m, rb + rpc);
  for (int r0 = rb; r0 < re; r0 += 32) {
    __syncthreads();
    double v[NBQ_MAX / 8];  // all of this thread's loads in flight before the stores
    const int r = r0 + (tid & 31);
#pragma unroll
    for (int u = 0; u < NBQ_MAX / 8; u++) {
      const int c = (tid >> 5) + 8 * u;
      v[u] = 0.0;
      if (r < re && c < ncol) v[u] = c < kb ? leaf_v(L, lda, r, c) : L[r + (long)c * lda];
    }
#pragma unroll
    for (int u = 0; u < NBQ_MAX / 8; u++) {
      const int c = (tid >> 5) + 8 * u;
      if (c < ncol) X[c][tid & 31] = v[u];
    }
    __syncthreads();
    const int nr = min(32, re - r0);
    for (int rr = 0; rr < nr; rr++) {
      const double xa = a < kb ? X[a][rr] : 0.0;
#pragma unroll
      for (int j = 0; j < NJ; j++) {
        const int b = b0 + SB * j;
        if (b < ncol) acc[j] = fma(xa, X[b][rr], acc[j]);
      }
    }
  }
  double *P = part + (size_t)blockIdx.x * QL_OUT;
#pragma unroll
  for (int j = 0; j < NJ; j++) P[a + (b0 + SB * j) * KB] = acc[j];
}

// P[o] = sum over g < ngrid of part[g][o], o < nout: eight partial sums per
// output (warps), combined in a fixed order
__global__ void __launch_bounds__(256) qr_leaf_reduce_kernel(int ngrid, int nout, const double *part, double *P) {
  __shared__ double red[8][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, o = blockIdx.x * 32 + lane;
  double v = 0.0;
  if (o < nout)
    for (int g = w; g < ngrid; g += 8) v += part[(size_t)g * QL_OUT + o];
  red[w][lane] = v;
  __syncthreads();
  if (w == 0 && o < nout) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) t += red[q][lane];
    P[o] = t;
  }
}

template <int KB>
__global__ void __launch_bounds__(256) qr_leaf_apply_kernel(int m, int kb, int n2, double *L, long lda,
                                                            const double *P, const double *tau) {
  constexpr int RPT = KB == 8 ? 4 : 2;  // rows per thread
  __shared__ double sT[KB][KB + 1];
  __shared__ double sW[KB][NBQ_MAX + 1];  // W = V^T C, then Y = T^T W in its place
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int base = 0; base < KB * (kb + n2); base += 256 * 8) {  // eight loads in flight per thread
    const int tot = KB * (kb + n2);
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, a = idx % KB;
      v[u] = (idx < tot && a < kb) ? P[idx] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * 256 + tid, a = idx % KB, b = idx / KB;
      if (idx >= tot) continue;
      if (b < kb) sT[a][b] = v[u];  // G = V^T V for now
      else sW[a][b - kb] = v[u];
    }
  }
  __syncthreads();
  if (w == 0) {  // T from G (upper; the recurrence overwrites G's strictly upper part)
    for (int i = 0; i < kb; i++) {
      double val = 0.0;
      if (lane < i) {
        for (int q = lane; q < i; q++) val = fma(sT[lane][q], sT[q][i], val);
        val *= -tau[i];
      }
      __syncwarp();
      if (lane < i) sT[lane][i] = val;
      if (lane == i) sT[i][i] = tau[i];
      __syncwarp();
    }
  }
  __syncthreads();
  constexpr int NY = KB * NBQ_MAX / 256;  // Y = T^T W: outputs per thread, held until W is read
  double y[NY];
#pragma unroll
  for (int u = 0; u < NY; u++) {
    const int idx = tid + 256 * u, a = idx % KB, c = idx / KB;
    double v = 0.0;
    if (a < kb && c < n2)
      for (int q = 0; q <= a; q++) v = fma(sT[q][a], sW[q][c], v);
    y[u] = v;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < NY; u++) {
    const int idx = tid + 256 * u;
    sW[idx % KB][idx / KB] = y[u];
  }
  __syncthreads();
  // C -= V Y: 32 lanes x RPT rows by 8 column groups per CTA tile of 32 * RPT rows
  const int cq = w;
  for (int rt = blockIdx.x * 32 * RPT; rt < m; rt += gridDim.x * 32 * RPT) {
    double v[RPT][KB];
#pragma unroll
    for (int i = 0; i < RPT; i++) {
      const int r = rt + lane + 32 * i;
#pragma unroll
      for (int a = 0; a < KB; a++) v[i][a] = (r < m && a < kb) ? leaf_v(L, lda, r, a) : 0.0;
    }
#pragma unroll 2
    for (int c = cq; c < n2; c += 8) {
      double acc[RPT];
#pragma unroll
      for (int i = 0; i < RPT; i++) acc[i] = 0.0;
#pragma unroll
      for (int a = 0; a < KB; a++) {
        const double y = sW[a][c];
#pragma unroll
        for (int i = 0; i < RPT; i++) acc[i] = fma(v[i][a], y, acc[i]);
      }
#pragma unroll
      for (int i = 0; i < RPT; i++) {
        const int r = rt + lane + 32 * i;
        if (r < m) L[r + (long)(kb + c) * lda] -= acc[i];
      }
    }
  }
}

template <int KB>
void leaf_apply_t(int m, int kb, int n2, double *L, long lda, const double *tau, double *part, double *P,
                  cudaStream_t st) {
  const int ncol = kb + n2;
  const int rpc = cdiv(cdiv(m, QL_GRID), 32) * 32;
  const int grid = cdiv(m, rpc);
  qr_leaf_gram_kernel<KB><<<grid, 256, 0, st>>>(m, kb, ncol, L, lda, rpc, part);
  ATLB_CUDA_CHECK(cudaGetLastError());
  const int nout = KB * ncol;
  qr_leaf_reduce_kernel<<<cdiv(nout, 32), 256, 0, st>>>(grid, nout, part, P);
  ATLB_CUDA_CHECK(cudaGetLastError());
  constexpr int RPT = KB == 8 ? 4 : 2;
  const int agrid = std::min(cdiv(m, 32 * RPT), 2 * num_sms());
  qr_leaf_apply_kernel<KB><<<agrid, 256, 0, st>>>(m, kb, n2, L, lda, P, tau);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// the leaf at L (m x kb, factored) applied to the n2 columns on its right
void leaf_apply(int m, int kb, int n2, double *L, long lda, const double *tau, double *part, double *P,
                cudaStream_t st) {
  if (m <= 0 || n2 <= 0 || kb <= 0) return;
  if (kb <= 8) leaf_apply_t<8>(m, kb, n2, L, lda, tau, part, P, st);
  else if (kb <= 16) leaf_apply_t<16>(m, kb, n2, L, lda, tau, part, P, st);
  else leaf_apply_t<32>(m, kb, n2, L, lda, tau, part, P, st);
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

// V (m x k, explicit unit lower trapezoid of the factored panel at P),
// G = V^T V and T (k x k, ld k) of its block reflector.  k <= NBQ_MAX: one
// larft_kernel; k <= 2 NBQ_MAX (a panel of two halves): T of each half by
// larft_kernel, then T12 = -T1 (G12 T2) by two GEMMs (the same merge
// identity as inside larft_kernel), tmp holding G12 T2 (NBQ_MAX^2 doubles).
void build_vt(int m, int k, const double *P, long ldp, const double *tau, double *V, double *G,
              double *T, double *tmp, cudaStream_t st) {
  long tot = (long)m * k;
  extract_v_kernel<<<(int)std::min<long>((tot + 255) / 256, 8192), 256, 0, st>>>(m, k, P, ldp, V);
  ATLB_CUDA_CHECK(cudaGetLastError());
  dgemm_dev(kTrans, kNoTrans, k, k, m, 1.0, V, m, V, m, 0.0, G, k, st);
  static bool cfg = false;
  if (!cfg) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)larft_smem_bytes()));
    cfg = true;
  }
  if (k <= NBQ_MAX) {
    larft_kernel<<<1, 256, larft_smem_bytes(), st>>>(k, G, k, tau, T, k);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  const int k1 = NBQ_MAX, k2 = k - k1;
  double *T2 = T + k1 + (long)k1 * k;
  larft_kernel<<<1, 256, larft_smem_bytes(), st>>>(k1, G, k, tau, T, k);
  larft_kernel<<<1, 256, larft_smem_bytes(), st>>>(k2, G + k1 + (long)k1 * k, k, tau + k1, T2, k);
  ATLB_CUDA_CHECK(cudaGetLastError());
  ATLB_CUDA_CHECK(cudaMemset2DAsync(T + k1, sizeof(double) * k, 0, sizeof(double) * k2, k1, st));  // T21 = 0
  dgemm_dev(kNoTrans, kNoTrans, k1, k2, k2, 1.0, G + (long)k1 * k, k, T2, k, 0.0, tmp, k1, st);
  dgemm_dev(kNoTrans, kNoTrans, k1, k2, k1, -1.0, T, k, tmp, k1, 0.0, T + (long)k1 * k, k, st);
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
  size_t need = (size_t)nq * NBQ + 2 * (size_t)NBQ * NBQ + 2 * (size_t)NBQ * other + (size_t)NBQ_MAX * NBQ_MAX;
  double *ws = (double *)scratch(kSlotQrApply, sizeof(double) * need);
  double *V = ws, *G = V + (size_t)nq * NBQ, *T = G + (size_t)NBQ * NBQ, *W = T + (size_t)NBQ * NBQ;
  double *tmp = W + 2 * (size_t)NBQ * other;
  const int nblk = cdiv(K, NBQ);
  // Q C = H0 (H1 (... C)): last block first; Q^T C: first block first (Left).
  // C Q = ((C H0) H1) ...: first block first; C Q^T: last block first (Right).
  const bool forward = (side == kLeft) == (trans != kNoTrans);
  for (int t = 0; t < nblk; t++) {
    const int b = forward ? t : nblk - 1 - t;
    const int j = b * NBQ, kb = std::min(NBQ, K - j), len = nq - j;
    build_vt(len, kb, A + j + (long)j * lda, lda, tau + j, V, G, T, tmp, st);
    if (side == kLeft) larfb_gen(kLeft, trans, len, other, kb, V, T, C + j, ldc, W, st);
    else larfb_gen(kRight, trans, len, other, kb, V, T, C + (long)j * ldc, ldc, W, st);
  }
}

// Workspace of one stream's share of the factorization: V (M x NBQ), G and
// T (NBQ x NBQ), W (2 x NBQ x ncol), tmp (NBQ_MAX^2), the leaf passes'
// partial sums (QL_GRID x QL_OUT) and their total (QL_OUT).
struct QrWork {
  double *V, *G, *T, *W, *tmp, *part, *Psum;
};
size_t qr_work_doubles(int M, int NBQ, int ncol) {
  return (size_t)M * NBQ + 2 * (size_t)NBQ * NBQ + 2 * (size_t)NBQ * ncol + (size_t)NBQ_MAX * NBQ_MAX +
         (size_t)(QL_GRID + 1) * QL_OUT;
}
QrWork qr_work(double *ws, int M, int NBQ, int ncol) {
  QrWork w;
  w.V = ws;
  w.G = w.V + (size_t)M * NBQ;
  w.T = w.G + (size_t)NBQ * NBQ;
  w.W = w.T + (size_t)NBQ * NBQ;
  w.tmp = w.W + 2 * (size_t)NBQ * ncol;
  w.part = w.tmp + (size_t)NBQ_MAX * NBQ_MAX;
  w.Psum = w.part + (size_t)QL_GRID * QL_OUT;
  return w;
}

// Factor the m x nb panel at P.  Up to NBQ_MAX columns: leaves, each applied
// to the panel's columns on its right (the reference's recursive panel
// ATL_geqrr).  Wider (up to 2 NBQ_MAX): the left half so, its block
// reflector applied to the right half (larfb, K = NBQ_MAX), then the right
// half -- one more level of the same recursion.
void factor_panel(int m, int nb, double *P, long lda, double *tau, const QrWork &w, cudaStream_t st) {
  if (nb > NBQ_MAX) {
    const int h = NBQ_MAX;
    factor_panel(m, h, P, lda, tau, w, st);
    build_vt(m, h, P, lda, tau, w.V, w.G, w.T, w.tmp, st);
    larfb_lt(m, nb - h, h, w.V, w.T, P + (long)h * lda, lda, w.W, st);
    factor_panel(m - h, nb - h, P + h + (long)h * lda, lda, tau + h, w, st);
    return;
  }
  for (int l = 0; l < nb;) {
    const int leaf = std::min(qr_leaf(m - l), nb - l);
    double *L = P + l + (long)l * lda;
    geqr2_leaf(m - l, leaf, L, lda, tau + l, st);
    if (l + leaf < nb) leaf_apply(m - l, leaf, nb - l - leaf, L, lda, tau + l, w.part, w.Psum, st);
    l += leaf;
  }
}

void dgeqrf_dev(int M, int N, double *A, long lda, double *tau, cudaStream_t st) {
  const int mn = std::min(M, N);
  if (mn <= 0) return;
  const int NBQ = tune(kTuneQrNB);  // the outer panel width (ATL_ilaenv's NB, tuned; <= 2 NBQ_MAX)
  double *ws = (double *)scratch(kSlotWork, sizeof(double) * qr_work_doubles(M, NBQ, N));
  const QrWork w = qr_work(ws, M, NBQ, N);
  if (!lookahead_enabled() || mn <= NBQ) {
    for (int j = 0; j < mn; j += NBQ) {
      const int nb = std::min(NBQ, mn - j), m = M - j;
      double *P = A + j + (long)j * lda;
      factor_panel(m, nb, P, lda, tau + j, w, st);
      if (j + nb < N) {
        build_vt(m, nb, P, lda, tau + j, w.V, w.G, w.T, w.tmp, st);
        larfb_lt(m, N - j - nb, nb, w.V, w.T, P + (long)nb * lda, lda, w.W, st);
      }
    }
    return;
  }
  // Look-ahead of depth one (as in getrf and potrf): panel k's block
  // reflector updates panel k+1's columns first; the side stream factors
  // panel k+1 while the main stream updates the columns right of it.  The
  // side stream writes only panel k+1 (and its tau), the main stream only
  // the columns beyond it; the main stream's V is its own copy of panel k,
  // and the side stream has its own workspace (SideScope).
  cudaStream_t s1 = side_stream();
  QrWork sw;
  {
    SideScope side;
    double *sws = (double *)scratch(kSlotWork, sizeof(double) * qr_work_doubles(M, NBQ, NBQ));
    sw = qr_work(sws, M, NBQ, NBQ);
  }
  factor_panel(M, std::min(NBQ, mn), A, lda, tau, w, st);
  int k = 0;
  for (int j = 0; j < mn; j += NBQ, k++) {
    const int nb = std::min(NBQ, mn - j), m = M - j, jn = j + nb;
    if (jn >= N) break;
    double *P = A + j + (long)j * lda;
    if (k > 0) ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + (k & 1)), 0));  // panel k factored
    build_vt(m, nb, P, lda, tau + j, w.V, w.G, w.T, w.tmp, st);
    if (jn >= mn) {  // no panel after this one: columns mn..N-1 only
      larfb_lt(m, N - jn, nb, w.V, w.T, P + (long)nb * lda, lda, w.W, st);
      break;
    }
    const int nbn = std::min(NBQ, mn - jn), rest = N - jn - nbn;
    larfb_lt(m, nbn, nb, w.V, w.T, P + (long)nb * lda, lda, w.W, st);
    ATLB_CUDA_CHECK(cudaEventRecord(side_event(k & 1), st));
    ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(k & 1), 0));
    {
      SideScope side;
      factor_panel(M - jn, nbn, A + jn + (long)jn * lda, lda, tau + jn, sw, s1);
      ATLB_CUDA_CHECK(cudaEventRecord(side_event(2 + ((k + 1) & 1)), s1));
    }
    if (rest > 0) {
      const int reserve = tune(kTuneLookaheadReserve);
      GemmCtaCap cap(reserve > 0 ? std::max(1, num_sms() - reserve) : 0);
      larfb_lt(m, rest, nb, w.V, w.T, P + (long)(nb + nbn) * lda, lda, w.W, st);
    }
  }
  ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + (k & 1)), 0));  // join the last panel
}

}  // namespace atlb
