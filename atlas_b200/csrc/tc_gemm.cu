// Tensor-core GEMMs on the 5th-generation tensor cores (tcgen05 / TMEM).
//
//   D[m][n] = sum_k A[m][k] * B[n][k]     A: M x K, B: N x K, both K-major
//
// Kinds: kind::f16 with BF16 operands, kind::tf32 (FP32 operands), both with
// FP32 accumulation; kind::i8 (signed INT8 operands, exact INT32
// accumulation).  One CTA computes a 128 x BN tile: warp 0 streams 128-byte
// K-slabs of A and B into a STAGES-deep ring of 128B-swizzled shared-memory
// tiles with TMA (each CTA loads its own tiles), one thread of warp 1 issues tcgen05.mma into
// a TMEM accumulator and releases each stage with tcgen05.commit, and all
// four warps drain TMEM (tcgen05.ld 32x32b) into the epilogue.  Every
// mbarrier wait is bounded: on timeout the kernel records an error code in
// *err, stops, frees its TMEM and returns.
//
// Epilogues: FP32 column-major C = alpha*D + beta*C (optionally one triangle
// only), and the split-integer (Ozaki) accumulation C_fp64 += w * rs[m] *
// cs[n] * D_int32.
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "tc_gemm.h"

namespace atlb {
namespace tc {

constexpr int BM = 128;
constexpr int SLAB = 128;  // bytes of K per stage (one 128B swizzle atom row)
constexpr int THREADS = 128;

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bounded wait for phase `parity` of the barrier; false after ~timeout_ns.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t timeout_ns) {
  uint32_t ok = 0;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  if (ok) return true;
  const uint64_t t0 = globaltimer();
  while (true) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    if (ok) return true;
    if (globaltimer() - t0 > timeout_ns) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(map), "r"(c0), "r"(c1), "r"(bar) : "memory");
}

// SMEM matrix descriptor: K-major, 128B swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
  d |= (uint64_t)1 << 46;                  // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
  return d;
}

template <int KIND>
__device__ __forceinline__ void mma_issue(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                          uint32_t acc) {
  if (KIND == kKindBF16) {
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
  } else if (KIND == kKindTF32) {
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }"
        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
  } else {
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }"
        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
  }
}

template <int KIND, int BN>
__host__ __device__ constexpr uint32_t instr_desc() {
  // c_format [4,6): 1 = F32, 2 = S32; a/b format [7,10)/[10,13): BF16 = 1,
  // TF32 = 2, signed INT8 = 1; K-major A and B; N>>3 at [17,23); M>>4 at [24,29)
  return (uint32_t)((KIND == kKindI8 ? 2u : 1u) << 4) |
         (uint32_t)((KIND == kKindTF32 ? 2u : 1u) << 7) |
         (uint32_t)((KIND == kKindTF32 ? 2u : 1u) << 10) |
         (uint32_t)((BN >> 3) << 17) | (uint32_t)((BM >> 4) << 24);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// MS M-subtiles of BM rows per CTA: each k-step issues MS MMAs that share
// the stage's B tile, into MS accumulators side by side in TMEM (MS * BN
// columns); a 256 x 256 tile moves half the operand bytes per product of a
// 128 x 256 one.
//
// SPLIT (TF32 only): each operand row holds two planes of K elements, the
// TF32 high parts at columns [0, K) and the TF32 remainders at [K, 2K).  A
// stage carries both planes of A and of B, and each k-step issues the three
// products hi*hi, lo*hi and hi*lo into the one accumulator: the operands
// cross L2 once per plane instead of once per product.
template <int KIND, int BN, int STAGES, int EPI, int MS = 1, int SPLIT = 0>
__global__ void __launch_bounds__(THREADS, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               int M, int N, int K, EpiParams ep, int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned base for the swizzled tiles
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int BMT = BM * MS;  // rows of the CTA's tile
  static_assert(MS * BN <= 512, "TMEM holds 512 columns");
  static_assert(!SPLIT || KIND == kKindTF32, "split operands are TF32 pairs");
  constexpr int NP = SPLIT ? 2 : 1;  // planes per operand
  constexpr int NPROD = SPLIT ? 3 : 1;
  // stage: A plane 0 [, A plane 1], B plane 0 [, B plane 1], each 1024-byte aligned
  constexpr int A_BYTES = BMT * SLAB, B_BYTES = BN * SLAB, STAGE = NP * (A_BYTES + B_BYTES);
  uint64_t *bars = (uint64_t *)(smem + STAGES * STAGE);
  uint32_t *tmem_slot = (uint32_t *)(bars + 2 * STAGES + 1);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar_full = smem_u32(bars), bar_empty = bar_full + 8 * STAGES,
                 bar_done = bar_full + 16 * STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_n = (N + BN - 1) / BN;
  const int tm = blockIdx.x / tiles_n, tn = blockIdx.x % tiles_n;
  const int m0 = tm * BMT, n0 = tn * BN;
  if (EPI == kEpiF32 && ep.tri == 1 && m0 + BMT - 1 < n0) return;
  if (EPI == kEpiF32 && ep.tri == 2 && m0 > n0 + BN - 1) return;

  constexpr int ELEM = (KIND == kKindBF16) ? 2 : (KIND == kKindTF32 ? 4 : 1);
  constexpr int KPS = SLAB / ELEM;        // K elements per stage
  constexpr int KPM = 32 / ELEM;          // K elements per MMA instruction
  const int nkb = (K + KPS - 1) / KPS;
  const uint64_t TO = 2000000000ull;      // 2 s per wait

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {  // allocate MS * BN TMEM columns (power of two >= 32)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(tmem_slot)), "r"(MS * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (kb >= STAGES && !mbar_wait(bar_empty + 8 * s, ph ^ 1, TO)) { atomicExch(err, 1); break; }
      mbar_expect_tx(bar_full + 8 * s, STAGE);
#pragma unroll
      for (int p = 0; p < NP; p++) {
        tma_load_2d(sbase + s * STAGE + p * A_BYTES, &tmA, p * K + kb * KPS, m0, bar_full + 8 * s);
        tma_load_2d(sbase + s * STAGE + NP * A_BYTES + p * B_BYTES, &tmB, p * K + kb * KPS, n0,
                    bar_full + 8 * s);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    constexpr uint32_t idesc = instr_desc<KIND, BN>();
    bool ok = true;
    for (int kb = 0; kb < nkb; kb++) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (!mbar_wait(bar_full + 8 * s, ph, TO)) { atomicExch(err, 2); ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_addr = sbase + s * STAGE, b_addr = a_addr + NP * A_BYTES;
#pragma unroll
      for (int k = 0; k < KPS / KPM; k++) {
#pragma unroll
        for (int q = 0; q < NPROD; q++) {  // planes of (A, B): (0, 0), then (1, 0), (0, 1)
          const uint32_t pa = q == 1 ? A_BYTES : 0, pb = q == 2 ? B_BYTES : 0;
#pragma unroll
          for (int ms = 0; ms < MS; ms++)
            mma_issue<KIND>(tmem + ms * BN, smem_desc(a_addr + pa + ms * BM * SLAB + k * 32),
                            smem_desc(b_addr + pb + k * 32), idesc, (kb > 0 || k > 0 || q > 0) ? 1u : 0u);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(bar_empty + 8 * s) : "memory");
    }
    (void)ok;
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(bar_done) : "memory");
  }
  __syncwarp();

  // epilogue: every thread owns TMEM lane (= row) 32*warp + lane
  bool done = mbar_wait(bar_done, 0, 4 * TO);
  done = __all_sync(0xffffffffu, done);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!done) atomicExch(err, 3);
#pragma unroll 1
  for (int ms = 0; ms < MS; ms++) {
  const int m = m0 + ms * BM + warp * 32 + lane;
  if (done && nkb > 0) {
#pragma unroll 1
    for (int c = 0; c < BN / 32; c++) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + ms * BN + c * 32, r);
      if (m < M) {
        // all 32 old values of C first (independent loads, latencies overlap),
        // then the 32 results: the loads are not serialized behind the stores
        const int n1 = n0 + c * 32;
        if (EPI == kEpiF32) {
          float old[32];
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const int n = n1 + i;
            const bool ok = n < N && !(ep.tri == 1 && m < n) && !(ep.tri == 2 && m > n);
            old[i] = (ok && ep.beta != 0.f) ? ep.Cf[m + (long)n * ep.ldc] : 0.f;
          }
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const int n = n1 + i;
            const bool ok = n < N && !(ep.tri == 1 && m < n) && !(ep.tri == 2 && m > n);
            if (!ok) continue;
            float v = ep.alpha * __uint_as_float(r[i]);
            if (ep.beta != 0.f) v = fmaf(ep.beta, old[i], v);
            ep.Cf[m + (long)n * ep.ldc] = v;
          }
        } else {
          const double wr = ep.w * ep.rs[m];
          double old[32];
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const int n = n1 + i;
            old[i] = n < N ? ep.Cd[m + (long)n * ep.ldc] : 0.0;
          }
#pragma unroll
          for (int i = 0; i < 32; i++) {
            const int n = n1 + i;
            if (n < N) ep.Cd[m + (long)n * ep.ldc] = fma(wr * ep.cs[n], (double)(int)r[i], old[i]);
          }
        }
      }
    }
  } else if (nkb == 0 && EPI == kEpiF32 && m < M) {  // K == 0: C = beta*C
    for (int n = n0; n < min(N, n0 + BN); n++) {
      if (ep.tri == 1 && m < n) continue;
      if (ep.tri == 2 && m > n) continue;
      float *p = ep.Cf + m + (long)n * ep.ldc;
      *p = ep.beta == 0.f ? 0.f : ep.beta * *p;
    }
  }
  }  // M-subtiles
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MS * BN));
  }
}

// ---------------------------------------------------------------- host side

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    ATLB_CUDA_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess) {
      fprintf(stderr, "atlas_b200: cuTensorMapEncodeTiled unavailable\n");
      exit(-1);
    }
    fn = (EncodeTiledFn)p;
  }
  return fn;
}

// K-major rows x K operand, leading dimension ld elements (ld*elem % 16 == 0)
bool make_map(CUtensorMap *map, int kind, const void *base, int rows, int K, long ld, int box_rows) {
  const int elem = kind == kKindBF16 ? 2 : (kind == kKindTF32 ? 4 : 1);
  CUtensorMapDataType dt = kind == kKindBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                         : (kind == kKindTF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                              : CU_TENSOR_MAP_DATA_TYPE_UINT8);
  if (((uintptr_t)base % 16) || ((ld * elem) % 16)) return false;
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * elem)};
  cuuint32_t box[2] = {(cuuint32_t)(SLAB / elem), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(map, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int *err_flag() {
  static int *d = nullptr;
  if (!d) {
    ATLB_CUDA_CHECK(cudaMalloc(&d, sizeof(int)));
    ATLB_CUDA_CHECK(cudaMemset(d, 0, sizeof(int)));
  }
  return d;
}

// SPLIT: A and B rows hold two K-element planes (K a multiple of 32)
template <int KIND, int BN, int STAGES, int EPI, int MS = 1, int SPLIT = 0>
void launch_t(const void *A, long lda, const void *B, long ldb, int M, int N, int K,
              const EpiParams &ep, cudaStream_t st) {
  constexpr int NP = SPLIT ? 2 : 1;
  CUtensorMap ma, mb;
  if (!make_map(&ma, KIND, A, M, NP * K, lda, BM * MS) || !make_map(&mb, KIND, B, N, NP * K, ldb, BN)) {
    fprintf(stderr, "atlas_b200: tensor-map encoding failed (alignment)\n");
    set_cuda_error(cudaErrorInvalidValue);
    return;
  }
  constexpr int smem = STAGES * NP * (BM * MS + BN) * SLAB + 1024 + (2 * STAGES + 2) * 8 + 16;
  auto kern = tc_gemm_kernel<KIND, BN, STAGES, EPI, MS, SPLIT>;
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured = true;
  }
  const int tiles = cdiv(M, BM * MS) * cdiv(N, BN);
  kern<<<tiles, THREADS, smem, st>>>(ma, mb, M, N, K, ep, err_flag());
  ATLB_CUDA_CHECK(cudaGetLastError());
}

void tc_gemm(int kind, int epi, const void *A, long lda, const void *B, long ldb, int M, int N,
             int K, const EpiParams &ep, cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  if (kind == kKindBF16) {
    if (epi == kEpiF32) launch_t<kKindBF16, 128, 6, kEpiF32>(A, lda, B, ldb, M, N, K, ep, st);
  } else if (kind == kKindTF32) {
    // 128 x 64 tiles, 3 stages (73 KB of shared memory): the mixed solvers'
    // trailing updates leave room on each SM for the look-ahead stream's
    // kernels (measured: 2.5 % faster dsgesv than 128 x 128, 6 stages)
    if (epi == kEpiF32) launch_t<kKindTF32, 64, 3, kEpiF32>(A, lda, B, ldb, M, N, K, ep, st);
  } else {
    // 256 x 256 tiles (two 128-row accumulators): half the operand traffic
    // per product of 128 x 128 tiles
    if (epi == kEpiF64Acc) launch_t<kKindI8, 256, 3, kEpiF64Acc, 2>(A, lda, B, ldb, M, N, K, ep, st);
  }
}

// The split-TF32 product of two-plane operands (rows of 2 * ldk elements,
// ldk a multiple of 32).
void tc_gemm_split(const float *A2, const float *B2, long ldk, int M, int N, const EpiParams &ep,
                   cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  // 128 x 64 tiles, 2 stages of both planes (96 KB): two CTAs per SM, so one
  // CTA's epilogue runs under the other's products, and each CTA retires
  // after one tile, which keeps SMs turning over for the look-ahead stream
  launch_t<kKindTF32, 64, 2, kEpiF32, 1, 1>(A2, 2 * ldk, B2, 2 * ldk, M, N, (int)ldk, ep, st);
}

int read_and_clear_error(cudaStream_t st) {
  int h = 0;
  ATLB_CUDA_CHECK(cudaMemcpyAsync(&h, err_flag(), sizeof(int), cudaMemcpyDeviceToHost, st));
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  if (h) ATLB_CUDA_CHECK(cudaMemsetAsync(err_flag(), 0, sizeof(int), st));
  return h;
}

// ---------------------------------------------------------------- FP32 GEMM on tensor cores

// op(X) (rows x K) -> K-major copy: BF16, or FP32 rounded to TF32 (round to
// nearest, ties away), element (r, k) = trans ? X[r + k*ld] : X[k + r*ld]
// where `trans` means X is stored r-contiguous.
template <int KIND>
__global__ void to_kmajor_kernel(int rows, int K, const float *__restrict__ X, long ld, int rcontig,
                                 void *__restrict__ out, long ldo) {
  __shared__ float t[32][33];
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {  // the four loads in flight together
    const int j = ty + 8 * q;
    int r, k;
    if (rcontig) { r = r0 + tx; k = k0 + j; } else { k = k0 + tx; r = r0 + j; }
    v[q] = (r < rows && k < K) ? X[rcontig ? (r + (long)k * ld) : (k + (long)r * ld)] : 0.f;
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int j = ty + 8 * q;
    if (rcontig) t[j][tx] = v[q]; else t[tx][j] = v[q];  // t[k_local][r_local]
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int j = ty + 8 * q, r = r0 + j, k = k0 + tx;
    if (r < rows && k < K) {
      const float v = t[tx][j];
      if (KIND == kKindBF16) {
        ((unsigned short *)out)[k + (long)r * ldo] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      } else {
        uint32_t u;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
        ((float *)out)[k + (long)r * ldo] = __uint_as_float(u);
      }
    }
  }
}

// 3xTF32: op(X) -> rows of two K-planes, each ldk wide: the TF32-rounded
// high part hi(x) at [0, ldk) and the TF32-rounded remainder x - hi(x) at
// [ldk, 2 ldk).  The split GEMM sums hi*hi + lo*hi + hi*lo (the lo*lo term is
// below FP32 rounding); the tensor cores' FP32 accumulation then bounds the
// accuracy: measured against FP64, 2.3e-6 at K = 256 and 5.5e-5 at K = 8192,
// where FP32 FMA gives 4.2e-6.
struct SplitOperand {
  int rows, K;
  const float *X;
  long ld;
  int rcontig;  // X(r, k) at r + k*ld (else k + r*ld)
  float *out;
};
// Both operands of one GEMM in one launch: CTAs with blockIdx.y < ya convert
// A's 32 x 32 tiles, the others B's.  Each thread's four loads are issued
// before any is used.
__global__ void __launch_bounds__(256)
to_kmajor_split_kernel(SplitOperand opa, SplitOperand opb, int ya, long ldk) {
  __shared__ float t[32][33];
  const bool isa = (int)blockIdx.y < ya;
  const SplitOperand &op = isa ? opa : opb;
  const int r0 = (isa ? blockIdx.y : blockIdx.y - ya) * 32, k0 = blockIdx.x * 32;
  if (k0 >= op.K) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int j = ty + 8 * q;
    int r, k;
    if (op.rcontig) { r = r0 + tx; k = k0 + j; } else { k = k0 + tx; r = r0 + j; }
    v[q] = (r < op.rows && k < op.K) ? op.X[op.rcontig ? (r + (long)k * op.ld) : (k + (long)r * op.ld)] : 0.f;
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int j = ty + 8 * q;
    if (op.rcontig) t[j][tx] = v[q]; else t[tx][j] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int j = ty + 8 * q, r = r0 + j, k = k0 + tx;
    if (r < op.rows && k < op.K) {
      const float x = t[tx][j];
      uint32_t hi, lo;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
      const float rem = x - __uint_as_float(hi);
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(rem));
      float *o = op.out + (long)r * 2 * ldk + k;
      o[0] = __uint_as_float(hi);
      o[ldk] = __uint_as_float(lo);
    }
  }
}

void sgemm_tf32x3(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                  const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st, int tri) {
  if (M <= 0 || N <= 0) return;
  EpiParams ep = {};
  ep.Cf = C; ep.ldc = ldc; ep.alpha = alpha; ep.beta = beta; ep.tri = tri;
  if (K <= 0 || alpha == 0.f) {
    sgemm_dev(ta, tb, M, N, 0, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
    return;
  }
  // each K-plane padded to a whole 32-element TMA slab so the two planes line up
  const long ldk = (long)cdiv(K, 32) * 32;
  const size_t abytes = (size_t)M * 2 * ldk * 4, bbytes = (size_t)N * 2 * ldk * 4;
  unsigned char *buf = (unsigned char *)scratch(kSlotTc0, abytes + bbytes + 256);
  float *Ak = (float *)buf;
  float *Bk = (float *)(buf + ((abytes + 255) / 256) * 256);
  if (ldk != K) {  // zero the K padding once per call
    ATLB_CUDA_CHECK(cudaMemsetAsync(buf, 0, abytes + bbytes + 256, st));
  }
  const SplitOperand opa = {M, K, A, lda, ta == kNoTrans, Ak};
  const SplitOperand opb = {N, K, B, ldb, tb != kNoTrans, Bk};
  const int ya = cdiv(M, 32);
  to_kmajor_split_kernel<<<dim3(cdiv(K, 32), ya + cdiv(N, 32)), dim3(32, 8), 0, st>>>(opa, opb, ya, ldk);
  ATLB_CUDA_CHECK(cudaGetLastError());
  tc_gemm_split(Ak, Bk, ldk, M, N, ep, st);
}

template <int KIND>
void sgemm_tc(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
              const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st, int tri) {
  if (M <= 0 || N <= 0) return;
  EpiParams ep = {};
  ep.Cf = C; ep.ldc = ldc; ep.alpha = alpha; ep.beta = beta; ep.tri = tri;
  if (K <= 0 || alpha == 0.f) {
    sgemm_dev(ta, tb, M, N, 0, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
    return;
  }
  const int elem = KIND == kKindBF16 ? 2 : 4;
  const long ldk = (long)cdiv((long)K * elem, 16) * 16 / elem;
  const size_t abytes = (size_t)M * ldk * elem, bbytes = (size_t)N * ldk * elem;
  unsigned char *buf = (unsigned char *)scratch(kSlotTc0, abytes + bbytes + 256);
  void *Ak = buf;
  void *Bk = buf + ((abytes + 255) / 256) * 256;
  dim3 blk(32, 8);
  // A: op(A)(m,k) = ta ? A[k + m*lda] : A[m + k*lda]  (m-contiguous when not transposed)
  to_kmajor_kernel<KIND><<<dim3(cdiv(K, 32), cdiv(M, 32)), blk, 0, st>>>(M, K, A, lda, ta == kNoTrans, Ak, ldk);
  // B: op(B)(k,n) -> row n: tb ? B[n + k*ldb] (n-contiguous) : B[k + n*ldb]
  to_kmajor_kernel<KIND><<<dim3(cdiv(K, 32), cdiv(N, 32)), blk, 0, st>>>(N, K, B, ldb, tb != kNoTrans, Bk, ldk);
  ATLB_CUDA_CHECK(cudaGetLastError());
  tc_gemm(KIND, kEpiF32, Ak, ldk, Bk, ldk, M, N, K, ep, st);
}

}  // namespace tc

void sgemm_tf32_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                    const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                    int tri) {
  tc::sgemm_tc<tc::kKindTF32>(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}
void sgemm_tf32x3_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                      const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                      int tri) {
  tc::sgemm_tf32x3(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}
void sgemm_bf16_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                    const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                    int tri) {
  tc::sgemm_tc<tc::kKindBF16>(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}

}  // namespace atlb
