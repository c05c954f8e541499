// FP64 GEMM on the sm_100a FP64 tensor path (DMMA, mma.sync m8n8k4 f64).
//
// Replaces the amm micro-kernels + block copies of the reference GEMM driver
// (src/blas/ammm/ATL_ammm.c:12-364, ATL_iploops.c:19-181): instead of copying
// A/B into access-major blocks on the host, a 4-stage cp.async pipeline stages
// 128x16 tiles of op(A) and op(B) in shared memory in the layout their global
// memory already has (no transposing copy), and each of 8 warps accumulates a
// 64x32 block of C in registers with DMMA.  The same kernel computes one
// triangle of C for SYRK (tiles outside the triangle exit at once; elements
// outside it are not stored).
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "kernels.h"

namespace atlb {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, THREADS = 256, STAGES = 4, PAD = 4;

// Shared-memory layout of one operand tile of BO (outer) x BK.  "o" is the
// outer index (m for A, n for B), "k" the reduction index.  KC = the operand
// is k-contiguous in global memory (A transposed, B not transposed);
// otherwise o-contiguous.
template <bool KC, int BO> struct Lay;
template <int BO> struct Lay<false, BO> {
  static constexpr int LD = BO + PAD;  // 132 / 68 doubles (4 mod 16): conflict-free fragments
  static constexpr int SIZE = BK * LD;
  __device__ static __forceinline__ int at(int o, int k) { return k * LD + o; }
};
template <int BO> struct Lay<true, BO> {
  static constexpr int LD = BK + PAD;  // 20 doubles
  static constexpr int SIZE = BO * LD;
  __device__ static __forceinline__ int at(int o, int k) { return o * LD + k; }
};

// Issue the cp.async copies of one BO x BK tile (o0.., k0..) of an operand.
template <bool KC, int VEC, int BO>
__device__ __forceinline__ void load_tile(double *s, const double *X, long ld, int o0, int k0,
                                          int O, int K, int tid) {
  using L = Lay<KC, BO>;
  constexpr int N16 = BO * BK / 2 / THREADS, N8 = BO * BK / THREADS;  // copies per thread
  if (!KC) {
    if (VEC == 2) {
#pragma unroll
      for (int i = 0; i < N16; i++) {
        int c = tid + THREADS * i, k = c / (BO / 2), o = (c % (BO / 2)) * 2;
        int go = o0 + o, gk = k0 + k;
        double *d = s + L::at(o, k);
        const double *g = X + go + (long)gk * ld;
        if (gk < K && go + 1 < O) cp_async16(d, g, true);
        else {
          bool p0 = gk < K && go < O;
          cp_async8(d, p0 ? g : X, p0);
          cp_async8(d + 1, X, false);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < N8; i++) {
        int c = tid + THREADS * i, k = c / BO, o = c % BO;
        int go = o0 + o, gk = k0 + k;
        bool p = gk < K && go < O;
        cp_async8(s + L::at(o, k), p ? X + go + (long)gk * ld : X, p);
      }
    }
  } else {
    if (VEC == 2) {
#pragma unroll
      for (int i = 0; i < N16; i++) {
        int c = tid + THREADS * i, o = c >> 3, k = (c & 7) * 2;
        int go = o0 + o, gk = k0 + k;
        double *d = s + L::at(o, k);
        const double *g = X + gk + (long)go * ld;
        if (go < O && gk + 1 < K) cp_async16(d, g, true);
        else {
          bool p0 = go < O && gk < K;
          cp_async8(d, p0 ? g : X, p0);
          cp_async8(d + 1, X, false);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < N8; i++) {
        int c = tid + THREADS * i, o = c >> 4, k = c & 15;
        int go = o0 + o, gk = k0 + k;
        bool p = go < O && gk < K;
        cp_async8(s + L::at(o, k), p ? X + gk + (long)go * ld : X, p);
      }
    }
  }
}

// Tile shapes.  BNT = 128: 128 x 128 tiles, 4 stages, one CTA per SM (the
// long-K GEMMs).  BNT = 64: 128 x 64 tiles, 3 stages, two CTAs per SM, so
// that one CTA's epilogue (the old C tile in and the new one out) overlaps
// the other's main loop -- the short-K trailing updates of the
// factorizations (K = 128..256), where a 128 x 128 tile spends a large part
// of its time in the epilogue.
template <int BNT> struct TileCfg {
  static constexpr int STG = BNT == 128 ? STAGES : 3;
  static constexpr int MINB = BNT == 128 ? 1 : 2;
  static constexpr int WARPS_N = BNT / 32, WARPS_M = 8 / WARPS_N;
  static constexpr int WMT = BM / WARPS_M, MI = WMT / 8;  // warp tile: WMT x 32 = MI x 4 fragments
  template <bool TA, bool TB>
  static constexpr int smem_doubles() { return STG * (Lay<TA, BM>::SIZE + Lay<!TB, BNT>::SIZE); }
};
constexpr int SMALL_K = 256;  // K up to this uses the 128 x 64 tiles
// the grouped (batched) GEMM's tile width: its problems are small (K <= 512,
// M, N from 16), where the narrower tile wastes less on padding and two CTAs
// per SM overlap their epilogues
constexpr int GROUPED_BN = 64;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

// One BM x BNT tile of C = alpha*op(A)*op(B) + beta*C (column-major) at
// (m0, n0).  tri: 0 full, 1 lower (store row >= col), 2 upper (row <= col).
template <bool TA, bool TB, int VEC, int BNT = BN>
__device__ __forceinline__ void dgemm_tile(int M, int N, int K, double alpha, const double *__restrict__ A,
                                           long lda, const double *__restrict__ B, long ldb, double beta,
                                           double *__restrict__ C, long ldc, int tri, int m0, int n0,
                                           double *smem) {
  using CF = TileCfg<BNT>;
  constexpr int STG = CF::STG, MI = CF::MI;
  using LA = Lay<TA, BM>;     // A k-contiguous when transposed
  using LB = Lay<!TB, BNT>;   // B k-contiguous when not transposed
  double *sA = smem;
  double *sB = smem + STG * LA::SIZE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp % CF::WARPS_M) * CF::WMT, wn = (warp / CF::WARPS_M) * 32;

  double acc[MI][4][2];
#pragma unroll
  for (int i = 0; i < MI; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int KT = (K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STG - 1; s++) {
    if (s < KT) {
      load_tile<TA, VEC, BM>(sA + s * LA::SIZE, A, lda, m0, s * BK, M, K, tid);
      load_tile<!TB, VEC, BNT>(sB + s * LB::SIZE, B, ldb, n0, s * BK, N, K, tid);
    }
    cp_async_commit();
  }

  const int fr = lane >> 2, fk = lane & 3;
  for (int kt = 0; kt < KT; kt++) {
    cp_async_wait<STG - 2>();
    __syncthreads();
    {
      int nk = kt + STG - 1;
      if (nk < KT) {
        int st = nk % STG;
        load_tile<TA, VEC, BM>(sA + st * LA::SIZE, A, lda, m0, nk * BK, M, K, tid);
        load_tile<!TB, VEC, BNT>(sB + st * LB::SIZE, B, ldb, n0, nk * BK, N, K, tid);
      }
      cp_async_commit();
    }
    const double *a_s = sA + (kt % STG) * LA::SIZE;
    const double *b_s = sB + (kt % STG) * LB::SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double a[MI], b[4];
#pragma unroll
      for (int i = 0; i < MI; i++) a[i] = a_s[LA::at(wm + i * 8 + fr, kk + fk)];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = b_s[LB::at(wn + j * 8 + fr, kk + fk)];
#pragma unroll
      for (int i = 0; i < MI; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
    }
  }
  cp_async_wait<0>();

  // epilogue: C fragment row = lane>>2, cols = 2*(lane&3) + {0,1}.  With
  // beta != 0 the old C tile is first staged in shared memory (the pipeline
  // buffers are free now) by one burst of asynchronous copies, so its load
  // latency is paid once per tile rather than once per fragment row.
  auto ok = [&](int r, int c) {
    return r < M && c < N && !(tri == 1 && r < c) && !(tri == 2 && r > c);
  };
  constexpr int CLD = BM + 4;  // staged C: column-major, ld CLD (fits the pipeline buffers)
  static_assert(BNT * CLD <= STG * (Lay<false, BM>::SIZE + Lay<false, BNT>::SIZE), "C tile does not fit");
  double *sC = smem;
  if (beta != 0.0) {
    __syncthreads();  // every warp is done with the pipeline buffers
    for (int idx = tid; idx < BM * BNT; idx += THREADS) {
      const int rr = idx % BM, cc = idx / BM, r = m0 + rr, c = n0 + cc;
      if (ok(r, c)) cp_async8(sC + rr + cc * CLD, C + r + (long)c * ldc, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < MI; i++) {
    const int rr = wm + i * 8 + fr, r = m0 + rr;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int cc = wn + j * 8 + fk * 2 + h, c = n0 + cc;
        if (!ok(r, c)) continue;
        double v = alpha * acc[i][j][h];
        if (beta != 0.0) v = fma(beta, sC[rr + cc * CLD], v);
        C[r + (long)c * ldc] = v;
      }
  }
}

template <bool TA, bool TB, int VEC, int BNT>
__global__ void __launch_bounds__(THREADS, TileCfg<BNT>::MINB)
dgemm_dmma_kernel(int M, int N, int K, double alpha, const double *__restrict__ A, long lda,
                  const double *__restrict__ B, long ldb, double beta, double *__restrict__ C,
                  long ldc, int tri, int G) {
  extern __shared__ __align__(16) double smem[];
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (N + BNT - 1) / BNT;
  // grouped rasterisation: G tile-rows share B panels in L2
  const int bid = blockIdx.x;
  const int per_group = G * tiles_n, group = bid / per_group;
  const int first_m = group * G, gsz = min(tiles_m - first_m, G);
  const int tm = first_m + (bid % per_group) % gsz, tn = (bid % per_group) / gsz;
  const int m0 = tm * BM, n0 = tn * BNT;
  if (tri == 1 && m0 + BM - 1 < n0) return;
  if (tri == 2 && m0 > n0 + BNT - 1) return;
  dgemm_tile<TA, TB, VEC, BNT>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, m0, n0, smem);
}

// The same GEMM on a capped number of CTAs, each walking tiles t, t + grid,
// ... (same rasterisation): leaves SMs free for work on another stream
// (the factorizations' look-ahead panels).
template <bool TA, bool TB, int VEC>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_capped_kernel(int M, int N, int K, double alpha, const double *__restrict__ A, long lda,
                    const double *__restrict__ B, long ldb, double beta, double *__restrict__ C,
                    long ldc, int tri, int G) {
  extern __shared__ __align__(16) double smem[];
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (N + BN - 1) / BN, tiles = tiles_m * tiles_n;
  for (int bid = blockIdx.x; bid < tiles; bid += gridDim.x) {
    const int per_group = G * tiles_n, group = bid / per_group;
    const int first_m = group * G, gsz = min(tiles_m - first_m, G);
    const int tm = first_m + (bid % per_group) % gsz, tn = (bid % per_group) / gsz;
    const int m0 = tm * BM, n0 = tn * BN;
    if (tri == 1 && m0 + BM - 1 < n0) continue;
    if (tri == 2 && m0 > n0 + BN - 1) continue;
    dgemm_tile<TA, TB, VEC>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, m0, n0, smem);
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// Grouped (batched, uneven) GEMM: a persistent grid walks the 128x128 tiles
// of all problems; tile t belongs to problem order[p] where tile_start[p] <= t
// < tile_start[p+1] (problems sorted by decreasing size on the host).
template <bool TA, bool TB, int VEC, int BNT>
__global__ void __launch_bounds__(THREADS, TileCfg<BNT>::MINB)
dgemm_grouped_kernel(const GemmProb *__restrict__ probs, const int *__restrict__ order,
                     const int *__restrict__ tile_start, int count, int *__restrict__ next) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_t;
  const int total = tile_start[count];
  while (true) {
    if (threadIdx.x == 0) s_t = atomicAdd(next, 1);
    __syncthreads();
    const int t = s_t;
    if (t >= total) return;
    int lo = 0, hi = count - 1;  // last p with tile_start[p] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tile_start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const GemmProb pr = probs[order[lo]];
    const int local = t - tile_start[lo], tiles_n = (pr.N + BNT - 1) / BNT;
    const int m0 = (local / tiles_n) * BM, n0 = (local % tiles_n) * BNT;
    dgemm_tile<TA, TB, VEC, BNT>(pr.M, pr.N, pr.K, pr.alpha, pr.A, pr.lda, pr.B, pr.ldb, pr.beta, pr.C,
                                 pr.ldc, 0, m0, n0, smem);
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// Split-K for GEMMs with too few output tiles to fill the GPU (the small
// updates inside the factorizations): CTA (tile, s) multiplies over the s-th
// K range into its own dense partial P_s (ld = M); a second kernel sums the
// partials in a fixed order (deterministic) and applies alpha, beta and tri.
template <bool TA, bool TB, int VEC>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_splitk_kernel(int M, int N, int K, int kc, const double *__restrict__ A, long lda,
                    const double *__restrict__ B, long ldb, double *__restrict__ P) {
  extern __shared__ __align__(16) double smem[];
  const int tiles_m = (M + BM - 1) / BM;
  const int tm = blockIdx.x % tiles_m, tn = blockIdx.x / tiles_m, s = blockIdx.y;
  const int k0 = s * kc, kl = min(kc, K - k0);
  const double *As = TA ? A + k0 : A + (long)k0 * lda;
  const double *Bs = TB ? B + (long)k0 * ldb : B + k0;
  dgemm_tile<TA, TB, VEC>(M, N, kl, 1.0, As, lda, Bs, ldb, 0.0, P + (long)s * M * N, M, 0, tm * BM,
                          tn * BN, smem);
}

__global__ void splitk_reduce_kernel(int M, int N, int S, double alpha, const double *__restrict__ P,
                                     double beta, double *__restrict__ C, long ldc, int tri) {
  const long total = (long)M * N, mn = total;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % M), c = (int)(idx / M);
    if (tri == 1 && r < c) continue;
    if (tri == 2 && r > c) continue;
    double acc = 0.0;
    for (int s = 0; s < S; s++) acc += P[idx + s * mn];
    double *p = C + r + (long)c * ldc;
    double v = alpha * acc;
    if (beta != 0.0) v = fma(beta, *p, v);
    *p = v;
  }
}

__global__ void scale_kernel(int M, int N, double beta, double *C, long ldc, int tri) {
  long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  long total = (long)M * N;
  for (; idx < total; idx += (long)gridDim.x * blockDim.x) {
    int r = (int)(idx % M), c = (int)(idx / M);
    if (tri == 1 && r < c) continue;
    if (tri == 2 && r > c) continue;
    double *p = C + r + (long)c * ldc;
    *p = (beta == 0.0) ? 0.0 : beta * *p;
  }
}

// Slices for a split-K GEMM of `tiles` output tiles (too few for the SMs):
// the smallest count, slices of at least 2 BK, whose CTAs (tiles x slices)
// fill their waves of nsm within 3 % of the best count -- e.g. 63 tiles take
// 7 slices (441 CTAs in 3 full waves), not 3 (189 CTAs, a second wave of 41).
int splitk_count(int tiles, int K, int nsm) {
  const int smax = std::max(1, std::min(K / (2 * BK), 4 * nsm));
  auto fill = [&](int s) {
    const long c = (long)tiles * s;
    return (double)c / ((double)cdiv(c, (long)nsm) * nsm);
  };
  double best = 0.0;
  for (int s = 1; s <= smax; s++) best = std::max(best, fill(s));
  for (int s = 1; s <= smax; s++)
    if (fill(s) >= 0.97 * best) return s;
  return 1;
}

template <bool TA, bool TB, int VEC>
void launch(int M, int N, int K, double alpha, const double *A, long lda, const double *B,
            long ldb, double beta, double *C, long ldc, int tri, cudaStream_t st) {
  constexpr int smem = TileCfg<BN>::template smem_doubles<TA, TB>() * (int)sizeof(double);
  constexpr int smem_s = TileCfg<64>::template smem_doubles<TA, TB>() * (int)sizeof(double);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_dmma_kernel<TA, TB, VEC, BN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_dmma_kernel<TA, TB, VEC, 64>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_s));
    // the largest shared-memory carveout, so that two of these CTAs fit on an SM
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_dmma_kernel<TA, TB, VEC, 64>,
                                         cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    configured = true;
  }
  int tiles = cdiv(M, BM) * cdiv(N, BN);
  // too few tiles for the 148 SMs and a long K: split K (partials + reduction)
  const int nsm = num_sms();
  int S = 1;
  if (tune(kTuneSplitK) && tiles * 2 <= nsm && K >= 4 * BK && !no_alloc_active()) S = splitk_count(tiles, K, nsm);
  if (S > 1) {
    const int kc = cdiv(cdiv(K, S), BK) * BK;
    S = cdiv(K, kc);
    double *P = (double *)scratch(kSlotGemmSplit, sizeof(double) * (size_t)S * M * N);
    if (P) {
      static bool configured_s = false;
      if (!configured_s) {
        ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_splitk_kernel<TA, TB, VEC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        configured_s = true;
      }
      dgemm_splitk_kernel<TA, TB, VEC><<<dim3(tiles, S), THREADS, smem, st>>>(M, N, K, kc, A, lda, B, ldb, P);
      const long total = (long)M * N;
      splitk_reduce_kernel<<<(int)std::min<long>((total + 255) / 256, 148L * 8), 256, 0, st>>>(
          M, N, S, alpha, P, beta, C, ldc, tri);
      ATLB_CUDA_CHECK(cudaGetLastError());
      return;
    }
  }
  const int cap = gemm_cta_cap();
  if (cap > 0 && tiles > cap) {
    static bool configured_c = false;
    if (!configured_c) {
      ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_capped_kernel<TA, TB, VEC>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      configured_c = true;
    }
    dgemm_capped_kernel<TA, TB, VEC><<<cap, THREADS, smem, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                                 ldc, tri, tune(kTuneGemmGroup));
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  if (K <= SMALL_K) {
    dgemm_dmma_kernel<TA, TB, VEC, 64><<<cdiv(M, BM) * cdiv(N, 64), THREADS, smem_s, st>>>(
        M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, tune(kTuneGemmGroup));
  } else {
    dgemm_dmma_kernel<TA, TB, VEC, BN><<<tiles, THREADS, smem, st>>>(M, N, K, alpha, A, lda, B, ldb,
                                                                     beta, C, ldc, tri, tune(kTuneGemmGroup));
  }
  ATLB_CUDA_CHECK(cudaGetLastError());
}

inline bool al16(const void *p, long ld) { return ((uintptr_t)p % 16 == 0) && (ld % 2 == 0); }

}  // namespace

void dgemm_dev(int ta, int tb, int M, int N, int K, double alpha, const double *A, long lda,
               const double *B, long ldb, double beta, double *C, long ldc, cudaStream_t st,
               int tri) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0 || alpha == 0.0) {
    if (beta == 1.0) return;
    long total = (long)M * N;
    int blocks = (int)std::min<long>((total + 255) / 256, 148L * 16);
    scale_kernel<<<blocks, 256, 0, st>>>(M, N, beta, C, ldc, tri);
    ATLB_CUDA_CHECK(cudaGetLastError());
    return;
  }
  const bool tA = ta != kNoTrans, tB = tb != kNoTrans;
  const bool v2 = al16(A, lda) && al16(B, ldb);
#define ATLB_DG(TA_, TB_)                                                                 \
  if (v2) launch<TA_, TB_, 2>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, st);    \
  else launch<TA_, TB_, 1>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, tri, st);
  if (!tA && !tB) { ATLB_DG(false, false) }
  else if (!tA && tB) { ATLB_DG(false, true) }
  else if (tA && !tB) { ATLB_DG(true, false) }
  else { ATLB_DG(true, true) }
#undef ATLB_DG
}

namespace {
template <bool TA, bool TB, int VEC>
void launch_grouped(const GemmProb *probs, const int *order, const int *tile_start, int count,
                    int *next, cudaStream_t st) {
  constexpr int smem = TileCfg<GROUPED_BN>::template smem_doubles<TA, TB>() * (int)sizeof(double);
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_grouped_kernel<TA, TB, VEC, GROUPED_BN>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(dgemm_grouped_kernel<TA, TB, VEC, GROUPED_BN>,
                                         cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    configured = true;
  }
  dgemm_grouped_kernel<TA, TB, VEC, GROUPED_BN><<<num_sms() * TileCfg<GROUPED_BN>::MINB, THREADS, smem, st>>>(
      probs, order, tile_start, count, next);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

void dgemm_grouped_dev(int ta, int tb, const GemmProb *hp, int count, cudaStream_t st) {
  if (count <= 0) return;
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  auto work = [&](int i) { return (long)hp[i].M * hp[i].N * hp[i].K; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  std::vector<int> ts(count + 1, 0);
  bool v2 = true;
  for (int i = 0; i < count; i++) {
    const GemmProb &p = hp[order[i]];
    ts[i + 1] = ts[i] + ((p.M > 0 && p.N > 0) ? cdiv(p.M, BM) * cdiv(p.N, GROUPED_BN) : 0);
    v2 = v2 && al16(p.A, p.lda) && al16(p.B, p.ldb);
  }
  const size_t bytes = sizeof(GemmProb) * count + sizeof(int) * (2 * count + 1 + 16);
  unsigned char *d = (unsigned char *)scratch(kSlotBatch3, bytes);
  unsigned char *h = (unsigned char *)pinned(kSlotBatch3, bytes);
  memcpy(h, hp, sizeof(GemmProb) * count);
  memcpy(h + sizeof(GemmProb) * count, order.data(), sizeof(int) * count);
  memcpy(h + sizeof(GemmProb) * count + sizeof(int) * count, ts.data(), sizeof(int) * (count + 1));
  memset(h + sizeof(GemmProb) * count + sizeof(int) * (2 * count + 1), 0, sizeof(int) * 16);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
  const GemmProb *dp = (const GemmProb *)d;
  const int *dord = (const int *)(d + sizeof(GemmProb) * count);
  const int *dts = dord + count;
  int *next = (int *)(dts + count + 1);
  const bool tA = ta != kNoTrans, tB = tb != kNoTrans;
#define ATLB_GG(TA_, TB_)                                                     \
  if (v2) launch_grouped<TA_, TB_, 2>(dp, dord, dts, count, next, st);       \
  else launch_grouped<TA_, TB_, 1>(dp, dord, dts, count, next, st);
  if (!tA && !tB) { ATLB_GG(false, false) }
  else if (!tA && tB) { ATLB_GG(false, true) }
  else if (tA && !tB) { ATLB_GG(true, false) }
  else { ATLB_GG(true, true) }
#undef ATLB_GG
  // the host staging buffer must outlive the copy: wait for it here
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
}

}  // namespace atlb
