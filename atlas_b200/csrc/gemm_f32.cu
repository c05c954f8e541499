// FP32 GEMM on the FP32 FMA pipes (cblas_sgemm and the FP32-exact factor
// mode of the mixed-precision solvers).  128x128x8 CTA tile, 256 threads,
// 8x8 outputs per thread; op(A) and op(B) tiles are staged in shared memory
// k-major (m / n contiguous) by a 3-stage cp.async pipeline, whatever their
// global layout, so the inner loop reads 128-bit vectors.  An output of few
// tiles with a long K (the Cholesky's diagonal-block updates) is split along
// K over gridDim.y: each slice writes its partial product to a workspace and
// one pass sums the slices into C.
// Reference semantics: src/blas/reference/level3/ATL_srefgemm.c.
#include <cstdint>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int BM = 128, BN = 128, BK = 8, THREADS = 256, STAGES = 3, LDS = BM + 4;

template <bool TRANS_O>  // operand element (o, k): TRANS_O ? X[k + o*ld] : X[o + k*ld]
__device__ __forceinline__ void load_tile(float *s, const float *X, long ld, int o0, int k0,
                                          int O, int K, int tid) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int c = tid + THREADS * i;
    int o, k;
    if (!TRANS_O) { o = c & 127; k = c >> 7; }   // o fastest: coalesced along o
    else { k = c & 7; o = c >> 3; }              // k fastest: coalesced along k
    int go = o0 + o, gk = k0 + k;
    bool p = go < O && gk < K;
    const float *g = TRANS_O ? X + gk + (long)go * ld : X + go + (long)gk * ld;
    cp_async4(s + k * LDS + o, p ? g : X, p);
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(THREADS, 2)
sgemm_simt_kernel(int M, int N, int K, float alpha, const float *__restrict__ A, long lda,
                  const float *__restrict__ B, long ldb, float beta, float *__restrict__ C,
                  long ldc, int tri, int kc, float *__restrict__ W) {
  if (gridDim.y > 1) {  // K slice blockIdx.y: its partial product, unscaled, into W's slice (ld M)
    const int k0 = blockIdx.y * kc;
    A += TA ? (long)k0 : (long)k0 * lda;
    B += TB ? (long)k0 * ldb : (long)k0;
    K = min(kc, K - k0);
    C = W + (long)blockIdx.y * M * N;
    ldc = M;
    alpha = 1.f;
    beta = 0.f;
  }
  __shared__ __align__(16) float sA[STAGES][BK * LDS];
  __shared__ __align__(16) float sB[STAGES][BK * LDS];
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (N + BN - 1) / BN;
  const int bid = blockIdx.x, G = 8;
  const int per_group = G * tiles_n, group = bid / per_group;
  const int first_m = group * G, gsz = min(tiles_m - first_m, G);
  const int tm = first_m + (bid % per_group) % gsz, tn = (bid % per_group) / gsz;
  const int m0 = tm * BM, n0 = tn * BN;
  if (tri == 1 && m0 + BM - 1 < n0) return;
  if (tri == 2 && m0 > n0 + BN - 1) return;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

  const int KT = (K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < KT) {
      load_tile<TA>(sA[s], A, lda, m0, s * BK, M, K, tid);
      load_tile<!TB>(sB[s], B, ldb, n0, s * BK, N, K, tid);
    }
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; kt++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      int nk = kt + STAGES - 1;
      if (nk < KT) {
        load_tile<TA>(sA[nk % STAGES], A, lda, m0, nk * BK, M, K, tid);
        load_tile<!TB>(sB[nk % STAGES], B, ldb, n0, nk * BK, N, K, tid);
      }
      cp_async_commit();
    }
    const float *as = sA[kt % STAGES], *bs = sB[kt % STAGES];
#pragma unroll
    for (int k = 0; k < BK; k++) {
      float4 a0 = *reinterpret_cast<const float4 *>(as + k * LDS + ty * 4);
      float4 a1 = *reinterpret_cast<const float4 *>(as + k * LDS + 64 + ty * 4);
      float4 b0 = *reinterpret_cast<const float4 *>(bs + k * LDS + tx * 4);
      float4 b1 = *reinterpret_cast<const float4 *>(bs + k * LDS + 64 + tx * 4);
      float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
  }
  cp_async_wait<0>();
  // epilogue: each thread owns rows {ty*4 .. +3, 64 + ty*4 .. +3} x columns
  // {tx*4 .. +3, 64 + tx*4 .. +3}; a row quad of one column is contiguous in C.
  // All old C values are loaded before any store, so the loads overlap.
  const bool vec = tri == 0 && ((uintptr_t)C % 16 == 0) && (ldc % 4 == 0) && m0 + BM <= M && n0 + BN <= N;
  if (vec) {
#pragma unroll
    for (int jh = 0; jh < 8; jh += 4) {  // two rounds of 8 float4 loads, then their stores
      float4 cv[4][2];
#pragma unroll
      for (int jj = 0; jj < 4; jj++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int j = jh + jj;
          const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4), r = m0 + h * 64 + ty * 4;
          cv[jj][h] = beta != 0.f ? *reinterpret_cast<const float4 *>(C + r + (long)c * ldc)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
      for (int jj = 0; jj < 4; jj++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int j = jh + jj;
          const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4), r = m0 + h * 64 + ty * 4;
          float4 o;
          o.x = alpha * acc[h * 4 + 0][j];
          o.y = alpha * acc[h * 4 + 1][j];
          o.z = alpha * acc[h * 4 + 2][j];
          o.w = alpha * acc[h * 4 + 3][j];
          if (beta != 0.f) {
            o.x = fmaf(beta, cv[jj][h].x, o.x);
            o.y = fmaf(beta, cv[jj][h].y, o.y);
            o.z = fmaf(beta, cv[jj][h].z, o.z);
            o.w = fmaf(beta, cv[jj][h].w, o.w);
          }
          *reinterpret_cast<float4 *>(C + r + (long)c * ldc) = o;
        }
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
    float cv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
      const bool ok = r < M && c < N && !(tri == 1 && r < c) && !(tri == 2 && r > c);
      cv[i] = (ok && beta != 0.f) ? C[r + (long)c * ldc] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
      if (r >= M || c >= N) continue;
      if (tri == 1 && r < c) continue;
      if (tri == 2 && r > c) continue;
      float v = alpha * acc[i][j];
      if (beta != 0.f) v = fmaf(beta, cv[i], v);
      C[r + (long)c * ldc] = v;
    }
  }
}

// C = beta C + alpha (sum of the S partial products in W, ld M), in C's triangle
__global__ void splitk_sum_kernel(int M, int N, int S, const float *__restrict__ W, float alpha, float beta,
                                  float *__restrict__ C, long ldc, int tri) {
  const long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % M), c = (int)(idx / M);
    if (tri == 1 && r < c) continue;
    if (tri == 2 && r > c) continue;
    float v = 0.f;
    for (int s = 0; s < S; s++) v += W[idx + (long)s * total];
    float *p = C + r + (long)c * ldc;
    *p = beta == 0.f ? alpha * v : fmaf(beta, *p, alpha * v);
  }
}

__global__ void sscale_kernel(int M, int N, float beta, float *C, long ldc, int tri) {
  long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  long total = (long)M * N;
  for (; idx < total; idx += (long)gridDim.x * blockDim.x) {
    int r = (int)(idx % M), c = (int)(idx / M);
    if (tri == 1 && r < c) continue;
    if (tri == 2 && r > c) continue;
    float *p = C + r + (long)c * ldc;
    *p = (beta == 0.f) ? 0.f : beta * *p;
  }
}

}  // namespace

void sgemm_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
               const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
               int tri) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0 || alpha == 0.f) {
    if (beta == 1.f) return;
    long total = (long)M * N;
    int blocks = (int)std::min<long>((total + 255) / 256, 148L * 16);
    sscale_kernel<<<blocks, 256, 0, st>>>(M, N, beta, C, ldc, tri);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  int tiles = cdiv(M, BM) * cdiv(N, BN);
  const bool tA = ta != kNoTrans, tB = tb != kNoTrans;
  // few output tiles and a long K: split K so that about two CTAs per SM run
  int S = 1, kc = K;
  float *W = nullptr;
  if (tiles < num_sms() / 2 && K >= 1024 && !no_alloc_active()) {
    S = std::min(cdiv(K, 256), std::max(1, 2 * num_sms() / tiles));
    kc = cdiv(cdiv(K, S), BK) * BK;
    S = cdiv(K, kc);
    if (S > 1) W = (float *)scratch(kSlotGemmSplit, sizeof(float) * (size_t)S * M * N);
    else kc = K;
  }
  const dim3 grid(tiles, S);
  if (!tA && !tB) sgemm_simt_kernel<false, false><<<grid, THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, kc, W);
  else if (!tA && tB) sgemm_simt_kernel<false, true><<<grid, THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, kc, W);
  else if (tA && !tB) sgemm_simt_kernel<true, false><<<grid, THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, kc, W);
  else sgemm_simt_kernel<true, true><<<grid, THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, kc, W);
  ATLB_CUDA_CHECK(cudaGetLastError());
  if (S > 1) {
    const long total = (long)M * N;
    splitk_sum_kernel<<<(int)std::min<long>((total + 255) / 256, 148L * 8), 256, 0, st>>>(M, N, S, W, alpha, beta, C,
                                                                                      ldc, tri);
    ATLB_CUDA_CHECK(cudaGetLastError());
  }
}

}  // namespace atlb
