// LU factorization with partial pivoting (clapack_dgetrf / ATL_getrfC) and
// the solve (ATL_getrs).
//
// Driver: the reference's recursive column halving (src/lapack/ATL_getrfC.c:
// 277-301): factor the left half, swap + TRSM + GEMM-update the right half,
// factor it, back-apply its swaps to the left half.  The recursion stops at a
// panel of NB <= 32 columns, which ONE kernel factors: a thread-block cluster
// of up to 16 CTAs x 512 threads holds the panel's rows in registers (one
// row, or a few, per thread), and each column costs one cluster barrier:
// every CTA publishes its local pivot candidate (|value|, row position, and
// the candidate row itself) in shared memory, all CTAs read all candidates
// over distributed shared memory, pick the same winner (largest |value|,
// lowest row index on ties = cblas_idamax's first maximum, ATL_getf2.c:33),
// and update their own rows with it.  Row swaps are not performed during the
// panel: each row carries its current position and the final permutation is
// applied when the rows are written back.
#include <algorithm>
#include <type_traits>
#include <vector>
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

constexpr int PT = 512;  // threads per CTA of the panel kernel

template <typename T> __device__ __forceinline__ T safmin();
template <> __device__ __forceinline__ double safmin<double>() { return DBL_MIN; }
template <> __device__ __forceinline__ float safmin<float>() { return FLT_MIN; }

template <typename T, int NB>
struct PanelPub {  // one CTA's published candidate for one column
  T row[NB];
  T val;
  int pos;
};

// Factor the M x ncols panel at A (ncols <= NB, M >= ncols).  Writes
// ipiv[j] = roff + (pivot row within the panel) and atomically lowers
// *dinfo to roff + j + 1 for a zero pivot in column j.
template <typename T, int NB, int RPT>
__global__ void __launch_bounds__(PT, 1)
getf2_cluster_kernel(int M, int ncols, T *__restrict__ A, long lda, int *__restrict__ ipiv,
                     int roff, int *__restrict__ dinfo) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), crank = (int)cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int TOT = C * PT;
  const int MN = min(M, ncols);

  __shared__ PanelPub<T, NB> pub[2];
  __shared__ T grow[16][NB];
  __shared__ T gval[16];
  __shared__ int gpos[16];
  __shared__ T wval[PT / 32];
  __shared__ int wpos[PT / 32];

  T a[RPT][NB];
  int pos[RPT];
  bool act[RPT];
#pragma unroll
  for (int q = 0; q < RPT; q++) {
    int r = crank * PT + tid + q * TOT;
    act[q] = r < M;
    pos[q] = act[q] ? r : INT_MAX;
#pragma unroll
    for (int k = 0; k < NB; k++) a[q][k] = (act[q] && k < ncols) ? A[r + (long)k * lda] : T(0);
  }

  // publish this CTA's candidate for column c into pub[c & 1]
  auto publish = [&](int c) {
    T v = T(-1);
    int vp = INT_MAX;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
      if (act[q]) {
        T t = T(0);
#pragma unroll
        for (int k = 0; k < NB; k++)
          if (k == c) t = fabs(a[q][k]);
        if (t > v || (t == v && pos[q] < vp)) { v = t; vp = pos[q]; }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      T ov = __shfl_xor_sync(0xffffffffu, v, o);
      int op = __shfl_xor_sync(0xffffffffu, vp, o);
      if (ov > v || (ov == v && op < vp)) { v = ov; vp = op; }
    }
    if (lane == 0) { wval[warp] = v; wpos[warp] = vp; }
    __syncthreads();
    if (warp == 0) {
      v = lane < PT / 32 ? wval[lane] : T(-1);
      vp = lane < PT / 32 ? wpos[lane] : INT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        T ov = __shfl_xor_sync(0xffffffffu, v, o);
        int op = __shfl_xor_sync(0xffffffffu, vp, o);
        if (ov > v || (ov == v && op < vp)) { v = ov; vp = op; }
      }
      if (lane == 0) { pub[c & 1].val = v; pub[c & 1].pos = vp; }
    }
    __syncthreads();
    const int wp = pub[c & 1].pos;
#pragma unroll
    for (int q = 0; q < RPT; q++)
      if (act[q] && pos[q] == wp) {
#pragma unroll
        for (int k = 0; k < NB; k++) pub[c & 1].row[k] = a[q][k];
      }
    cl.sync();
  };

  if (MN > 0) publish(0);

  // The column loop is deliberately not unrolled (an unrolled NB x NB body
  // overflows the instruction cache); register rows are addressed through
  // compare-and-select over the NB columns instead.
#pragma unroll 1
  for (int j = 0; j < MN; j++) {
    const int b = j & 1;
    // gather every CTA's candidate (one distributed-shared-memory round trip)
    for (int idx = tid; idx < C * (NB + 2); idx += PT) {
      int r = idx / (NB + 2), e = idx % (NB + 2);
      PanelPub<T, NB> *rp = cl.map_shared_rank(&pub[b], r);
      if (e < NB) grow[r][e] = rp->row[e];
      else if (e == NB) gval[r] = rp->val;
      else gpos[r] = rp->pos;
    }
    __syncthreads();
    T best = T(-1);
    int p = INT_MAX, w = 0;
    for (int r = 0; r < C; r++) {
      T v = gval[r];
      int vp = gpos[r];
      if (v > best || (v == best && vp < p)) { best = v; p = vp; w = r; }
    }
    const T piv = grow[w][j];
    if (crank == 0 && tid == 0) {
      ipiv[j] = roff + p;
      if (piv == T(0)) atomicMin(dinfo, roff + j + 1);
    }
    const bool use_rcp = fabs(piv) >= safmin<T>();
    const T rcp = T(1) / piv;
    const T *u = grow[w];
#pragma unroll
    for (int q = 0; q < RPT; q++) {
      if (!act[q]) continue;
      if (pos[q] == p) {  // the pivot row becomes row j of U
        act[q] = false;
        pos[q] = j;
        continue;
      }
      if (pos[q] == j) pos[q] = p;  // the row displaced by the swap
      if (piv != T(0)) {
        T aj = T(0);
#pragma unroll
        for (int k = 0; k < NB; k++)
          if (k == j) aj = a[q][k];
        const T l = use_rcp ? aj * rcp : aj / piv;
#pragma unroll
        for (int k = 0; k < NB; k++) {
          if (k == j) a[q][k] = l;
          else if (k > j) a[q][k] = fma(-l, u[k], a[q][k]);
        }
      }
    }
    if (j + 1 < MN) publish(j + 1);
  }

  // write rows back at their final positions (the permutation is applied here)
#pragma unroll
  for (int q = 0; q < RPT; q++) {
    int r = crank * PT + tid + q * TOT;
    if (r < M) {
#pragma unroll
      for (int k = 0; k < NB; k++)
        if (k < ncols) A[pos[q] + (long)k * lda] = a[q][k];
    }
  }
  cl.sync();  // keep this CTA's shared memory alive until every peer is done
}

// Leaf panel kernel: LU with partial pivoting of an M x ncols panel (ncols
// <= 32, M <= 512 x cluster size), fused with the two operations that
// follow it inside a block column of the factorization:
//   * the panel's row interchanges applied to the block's other columns
//     (nleft columns left of the panel, nright right of it), and
//   * the triangular solve U12 = L11^-1 A12 of the right columns' top rows.
// One thread holds one row, SHIFTED: a[0] is always the current column, so
// the rank-1 update is a[k-1] = a[k] - l*u[k] over fixed register indices.
// Finished parts of rows go to shared memory (L multipliers as produced, the
// U part of a pivot row when chosen) and reach their final row at the end.
//
// Per column, one cluster barrier and no remote reads: each CTA reduces its
// candidates (warp arg-max, then one __syncthreads), the CTA winner first
// completes its own row update, and its warp PUSHES (|value|, position, row)
// into a slot of every CTA's shared memory; after the barrier every warp
// reduces the C local slots to the same global winner.  The rest of the
// rank-1 update runs between the barrier's arrive and wait, so the barrier
// latency hides behind it.  Slots are double-buffered by column parity.
// Pivot order: largest |value|, lowest current row position on ties (the
// first maximum, like cblas_idamax); a NaN entry ranks below every number.
// One CTA's candidate for one column as it lands in every CTA's shared
// memory: a whole number of 16-byte units, each sent by one st.async.
template <typename T>
using PivKey = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
template <typename T, int NB>
struct __align__(16) PanelSlot {
  T row[NB];
  PivKey<T> key;  // pivot_key of the candidate
  typename std::conditional<sizeof(T) == 8, long long, int>::type pos;
  T rcp;          // 1 / (candidate value), computed by the sender off the critical path
  T lm;           // the sender's pending multiplier: the row is row - lm * u (see below)
};

// Candidates are compared through one integer key: |value|'s bit pattern + 1
// (non-negative IEEE values order like their bit patterns), 0 for a NaN or
// for "no candidate"; ties go to the lowest row position.  A warp's arg-max
// is then three redux instructions instead of a shuffle tree.
template <typename T>
__device__ __forceinline__ unsigned long long pivot_key(T v) {
  const T t = fabs(v);
  if (!(t >= T(0))) return 0ull;
  if (sizeof(T) == 8) return (unsigned long long)__double_as_longlong((double)t) + 1ull;
  return (unsigned long long)__float_as_uint((float)t) + 1ull;
}
__device__ __forceinline__ void warp_argmax_key(unsigned &key, unsigned &pos) {  // FP32 keys fit 32 bits
  const unsigned m = __reduce_max_sync(0xffffffffu, key);
  pos = __reduce_min_sync(0xffffffffu, key == m ? pos : 0xffffffffu);
  key = m;
}
__device__ __forceinline__ void warp_argmax_key(unsigned long long &key, unsigned &pos) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool eq = hi == mhi && lo == mlo;
  pos = __reduce_min_sync(0xffffffffu, eq ? pos : 0xffffffffu);
  key = ((unsigned long long)mhi << 32) | mlo;
}

// Lane of the warp's largest key (lowest pos among equal keys).  Usually
// the high 32 bits of the largest key occur in one lane only: one redux and
// one ballot then settle it.
template <typename K>
__device__ __forceinline__ int warp_argmax_lane(K key, unsigned pos) {
  const unsigned hi = sizeof(K) == 8 ? (unsigned)((unsigned long long)key >> 32) : (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned m = __ballot_sync(0xffffffffu, hi == mhi);
  if ((m & (m - 1)) == 0) return __ffs(m) - 1;
  K k = key;
  unsigned p = pos;
  warp_argmax_key(k, p);
  return __ffs(__ballot_sync(0xffffffffu, key == k && pos == p)) - 1;
}

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
// one-way 16-byte store into another CTA's shared memory that completes a
// transaction on that CTA's mbarrier (no fence, no round trip)
__device__ __forceinline__ void st_async16(uint32_t addr, uint4 v, uint32_t mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];"
               ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(a), "r"(parity) : "memory");
  return ok != 0;
}

// U12 = L11^-1 A12 for the panel kernels: L11 = the unit lower MN x MN top
// of the factored panel, A12 the top MN rows of the right columns.  Warp gw
// of GW solves columns 4 gw .. 4 gw + 3, 4 (gw + GW) .. and so on: lane i
// holds row i of four columns and row i of L11, and x_i -= L[i][k] x_k runs
// for k = 0, 1, .. in order (forward substitution, x_k by shuffle), four
// independent chains at a time.  Out of line so its registers do not add to
// the panel loop's.
template <typename T, int NB>
__device__ __noinline__ void panel_u12_solve(int MN, int ncols, int nright, int gw, int GW, T *A, long lda) {
  const int lane = threadIdx.x & 31;
  T L[NB - 1];
#pragma unroll
  for (int k = 0; k < NB - 1; k++) L[k] = (k < lane && lane < MN) ? __ldcg(A + lane + (long)k * lda) : T(0);
  for (int c0 = 4 * gw; c0 < nright; c0 += 4 * GW) {
    T x[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      x[q] = (c0 + q < nright && lane < MN) ? __ldcg(A + lane + (long)(ncols + c0 + q) * lda) : T(0);
#pragma unroll
    for (int k = 0; k < NB - 1; k++) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const T xk = __shfl_sync(0xffffffffu, x[q], k);
        if (lane > k) x[q] = fma(-L[k], xk, x[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (c0 + q < nright && lane < MN) A[lane + (long)(ncols + c0 + q) * lda] = x[q];
  }
}

// Shifted rank-1 update of a register row: a[k-1] = a[k] - l * u[k] for
// k = kfirst..NB-1 (a[NB-1] = 0 when kfirst == 1 ... see callers), with u
// read from shared memory 16 bytes at a time (u 16-byte aligned).
template <typename T, int NB>
__device__ __forceinline__ void shift_update(T (&a)[NB], T l, const T *u, int kfirst) {
  if (sizeof(T) == 4) {
    const float4 *u4 = reinterpret_cast<const float4 *>(u);
#pragma unroll
    for (int q = 0; q < NB / 4; q++) {
      const float4 v = u4[q];
      const T w[4] = {(T)v.x, (T)v.y, (T)v.z, (T)v.w};
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int k = 4 * q + e;
        if (k >= 1 && k >= kfirst) a[k - 1] = fma(-l, w[e], a[k]);
      }
    }
  } else {
    const double2 *u2 = reinterpret_cast<const double2 *>(u);
#pragma unroll
    for (int q = 0; q < NB / 2; q++) {
      const double2 v = u2[q];
      const T w[2] = {(T)v.x, (T)v.y};
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int k = 2 * q + e;
        if (k >= 1 && k >= kfirst) a[k - 1] = fma(-l, w[e], a[k]);
      }
    }
  }
  a[NB - 1] = T(0);
}

// stage[k] = a[k + off] (k < NB, zero past the row), 16 bytes per store
template <typename T, int NB>
__device__ __forceinline__ void stage_row(T *stage, const T (&a)[NB], int off) {
  if (sizeof(T) == 4) {
#pragma unroll
    for (int q = 0; q < NB / 4; q++) {
      float4 v;
      v.x = (float)(4 * q + 0 + off < NB ? a[(4 * q + 0 + off) % NB] : T(0));
      v.y = (float)(4 * q + 1 + off < NB ? a[(4 * q + 1 + off) % NB] : T(0));
      v.z = (float)(4 * q + 2 + off < NB ? a[(4 * q + 2 + off) % NB] : T(0));
      v.w = (float)(4 * q + 3 + off < NB ? a[(4 * q + 3 + off) % NB] : T(0));
      reinterpret_cast<float4 *>(stage)[q] = v;
    }
  } else {
#pragma unroll
    for (int q = 0; q < NB / 2; q++) {
      double2 v;
      v.x = (double)(2 * q + 0 + off < NB ? a[(2 * q + 0 + off) % NB] : T(0));
      v.y = (double)(2 * q + 1 + off < NB ? a[(2 * q + 1 + off) % NB] : T(0));
      reinterpret_cast<double2 *>(stage)[q] = v;
    }
  }
}

constexpr int kMaxPanelCluster = 16;
__device__ int g_panel_timeout = 0;  // set if a panel wait ever gives up (1 s)

template <typename T, int NB>
__global__ void __launch_bounds__(PT, 1)
getf2_fused_kernel(int M, int ncols, T *__restrict__ A, long lda, int *__restrict__ ipiv, int roff,
                   int *__restrict__ dinfo, int nleft, int nright) {
  static_assert(NB == 32, "one pivot-row element per lane");
  using Slot = PanelSlot<T, NB>;
  using K = PivKey<T>;
  constexpr int kUnits = (int)sizeof(Slot) / 16;  // 16-byte messages one CTA sends one CTA
  static_assert(sizeof(Slot) % 16 == 0, "slots travel as 16-byte units");
  constexpr uint32_t kMsg = sizeof(Slot);
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), crank = (int)cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int MN = min(M, ncols);
  extern __shared__ __align__(16) unsigned char fused_smem[];
  T *Lsm = reinterpret_cast<T *>(fused_smem);  // [NB][PT]: finished row parts
  __shared__ Slot slot[2][kMaxPanelCluster];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ __align__(16) T wu[2][PT / 32][NB];  // per-warp copy of the pivot row, by column parity
  __shared__ Slot stage;                       // the CTA winner's message
  __shared__ __align__(16) T zrow[NB];
  __shared__ K wv[2][PT / 32];                 // per-warp candidates, by column parity
  __shared__ unsigned wp[2][PT / 32];
  __shared__ int s_nmoved;
  __shared__ int s_from[2 * NB], s_to[2 * NB];  // rows that move: from (old) -> to (final)
  const uint32_t mb0 = smem_u32(&mbar[0]), mb1 = smem_u32(&mbar[1]);
  if (tid < NB) zrow[tid] = T(0);
  if (tid == 0) {
    s_nmoved = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  cluster_arrive();  // every CTA's barriers exist before anyone sends
  cluster_wait();

  const int r = crank * PT + tid;
  bool act = r < M;
  int pos = r;
  T a[NB];
  {
    const T *src = A + (act ? r : 0);
#pragma unroll
    for (int k = 0; k < NB; k++) {
      a[k] = (act && k < ncols) ? __ldg(src) : T(0);
      if (k + 1 < ncols) src += lda;
    }
  }
  T lm = T(0);
  const T *u = zrow;

  // Reduce this CTA's candidates (|a[0]| of active rows) and let the
  // winner's warp send its row for column c to every CTA's slot.  Inside the
  // column loop the winner has updated only a[0] (the candidate itself): it
  // sends row[0] = a[0] and row[1] (the next column, finished here with the
  // pivot row's u2) ready to use, its other entries as they are, shifted,
  // with its multiplier lm, and the receivers finish the update
  // (row[k] - lm * u[k+1], k >= 2) themselves, so the message leaves before
  // the sender's own row update.
  auto push = [&](int c, bool shifted, T u2) {
    const int b = c & 1;
    const uint32_t mb = b ? mb1 : mb0;
    if (tid == 0)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(kMsg * C) : "memory");
    const K v = act ? (K)pivot_key(a[0]) : K(0);
    const unsigned p = act ? (unsigned)pos : 0xffffffffu;
    const int wl = warp_argmax_lane(v, p);
    if (lane == wl) { wv[b][warp] = v; wp[b][warp] = p; }
    __syncthreads();
    const int wc = warp_argmax_lane(lane < PT / 32 ? wv[b][lane] : K(0),
                                    lane < PT / 32 ? wp[b][lane] : 0xffffffffu);
    if (warp == wc) {  // the warp of the CTA's candidate (or, without one, of a key that never wins)
      const bool owner = act && lane == wl;
      if (owner) {
        stage_row<T, NB>(stage.row, a, shifted ? 1 : 0);
        if (shifted) {
          stage.row[0] = a[0];
          stage.row[1] = fma(-lm, u2, a[2]);
        }
        stage.key = v;
        stage.pos = (int)p;
        stage.rcp = T(1) / a[0];
        stage.lm = shifted ? lm : T(0);
      }
      if (!__any_sync(0xffffffffu, owner) && lane == 0) {
        stage.key = K(0);
        stage.pos = -1;
      }
    }
    // kUnits x C messages of 16 bytes, at most one per thread
    static_assert(kUnits * kMaxPanelCluster <= PT, "one message per thread");
    __syncthreads();
    if (tid < kUnits * C) {
      const int q = tid / kUnits, unit = tid - q * kUnits;
      st_async16(mapa_u32(smem_u32(&slot[b][crank]) + 16 * unit, q), reinterpret_cast<const uint4 *>(&stage)[unit],
                 mapa_u32(mb, q));
    }
  };
  // wait until column c's C messages are in this CTA's slots
  auto receive = [&](int c) {
    const uint32_t mb = (c & 1) ? mb1 : mb0, parity = (c >> 1) & 1;
    if (!mbar_try_wait(mb, parity)) {
      uint64_t t0, t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
      while (!mbar_try_wait(mb, parity)) {
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 1000000000ull) { atomicExch(&g_panel_timeout, 1); break; }
      }
    }
  };

  if (MN > 0) {
    push(0, false, T(0));
    receive(0);
  }
  bool nz_prev = false;  // pivot of the previous column non-zero (its row is then the update row)
  bool piv_row = false;  // this row was chosen as a pivot (at column pos)
#pragma unroll 1
  for (int j = 0; j < MN; j++) {
    const int b = j & 1;
    // the global winner from the C local slots (every warp computes it)
    const unsigned mypos = lane < C ? (unsigned)slot[b][lane].pos : 0xffffffffu;
    const int w = warp_argmax_lane(lane < C ? slot[b][lane].key : K(0), mypos);
    const int p = (int)__shfl_sync(0xffffffffu, mypos, w);
    // the pivot, the next column's update coefficient and 1/pivot come ready
    // in the winner's slot; u2 (the pivot row's next entry) is for the next
    // sender
    const T *uprev = nz_prev ? wu[b ^ 1][warp] : zrow;
    const T piv = slot[b][w].row[0], u1 = slot[b][w].row[1], prcp = slot[b][w].rcp;
    const T lmw = slot[b][w].lm;
    const T u2 = fma(-lmw, uprev[3], slot[b][w].row[2]);
    {
      // the winner's full row for the rest of the update (lanes 0 and 1 came
      // finished), taken out of the slot before this column's message goes
      // out (after it, a CTA that has all of it may send column j + 2 here)
      const T rw = slot[b][w].row[lane];
      const T up = (lane >= 2 && lane < NB - 1) ? uprev[lane + 1] : T(0);
      wu[b][warp][lane] = lane < 2 ? rw : fma(-lmw, up, rw);
    }
    const bool nz = piv != T(0);
    if (crank == 0 && tid == 0) {
      ipiv[j] = roff + p;
      if (!nz) atomicMin(dinfo, roff + j + 1);
    }
    if (act) {
      if (pos == p) {  // this row becomes row j of U: its remaining part is final
        act = false;     // (stored after the loop, off the critical path)
        piv_row = true;
        pos = j;
      } else {
        if (pos == j) pos = p;  // the row displaced by the interchange
        // a zero pivot leaves the column unscaled and the row unchanged: the
        // update then runs with l = 0 against a zero row (exact: a - 0*0 = a)
        T l;
        if (!nz) l = a[0];
        else if (fabs(piv) >= safmin<T>()) l = a[0] * prcp;
        else l = a[0] / piv;
        lm = nz ? l : T(0);
        a[0] = fma(-lm, nz ? u1 : T(0), a[1]);  // the next column first: it decides the next pivot
        Lsm[j * PT + tid] = l;
        A[r + (long)j * lda] = l;  // at the row's original place (moved rows are rewritten at the end)
      }
    }
    if (j + 1 < MN) push(j + 1, true, nz ? u2 : T(0));
    __syncwarp();
    nz_prev = nz;
    u = nz ? wu[b][warp] : zrow;
    if (j + 1 < MN) {
      if (act) shift_update<T, NB>(a, lm, u, 2);  // it runs while the messages travel
      receive(j + 1);
    }
  }

  if (piv_row) {  // the U part of a pivot row: columns pos.. of the panel
    T *dst = Lsm + pos * PT + tid;
#pragma unroll
    for (int k = 0; k < NB; k++)
      if (pos + k < ncols) dst[k * PT] = a[k];
  }
  // Rows that moved register (from, to) in CTA 0's list, for the block's
  // other columns.  After one cluster barrier (which also orders the
  // multipliers stored during the loop before what follows), a row that
  // moved writes its whole panel row at its final place, a pivot row that
  // stayed its U part.
  const bool in = r < M;
  const int nother = nleft + nright;
  if (nother > 0 && in && pos != r) {
    int *cnt0 = cl.map_shared_rank(&s_nmoved, 0);
    const int i = atomicAdd(cnt0, 1);
    if (i < 2 * NB) {
      cl.map_shared_rank(s_from, 0)[i] = r;
      cl.map_shared_rank(s_to, 0)[i] = pos;
    }
  }
  __syncwarp();
  cluster_arrive();
  cluster_wait();
  if (in && (pos != r || piv_row)) {
    const int k0 = pos != r ? 0 : pos;
    for (int k = k0; k < ncols; k++) A[pos + (long)k * lda] = Lsm[k * PT + tid];
  }
  if (nother == 0) return;
  // The block's other columns of the rows that moved (at most 2*MN rows):
  // CTA q takes an equal share of the columns, reads the moved rows' old
  // values into shared memory and writes them to their final rows.
  __shared__ int l_from[2 * NB], l_to[2 * NB];
  const int nm = min(*cl.map_shared_rank(&s_nmoved, 0), 2 * NB);
  if (tid < nm) {
    l_from[tid] = cl.map_shared_rank(s_from, 0)[tid];
    l_to[tid] = cl.map_shared_rank(s_to, 0)[tid];
  }
  __syncthreads();  // the list is here and Lsm is free
  // CTA 0's shared memory must outlive the other CTAs' reads of its list: a
  // cluster barrier follows them before any CTA exits
  const bool u12 = nright > 0 && MN > 1;
  if (!u12) cluster_arrive();
  const int per = (nother + C - 1) / C, g0 = crank * per, ncol = max(0, min(nother, g0 + per) - g0);
  const int total = nm * ncol;  // <= 2 NB x NB*PT/(2 NB): fits Lsm
  for (int base = tid; base < total; base += 4 * PT) {
    T v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int g = base + q * PT;
      if (g < total) {
        const int i = g % nm, c = g0 + g / nm;
        const int col = c < nleft ? c - nleft : ncols + (c - nleft);
        v[q] = __ldcg(A + l_from[i] + (long)col * lda);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (base + q * PT < total) Lsm[base + q * PT] = v[q];
  }
  __syncthreads();
  for (int g = tid; g < total; g += PT) {
    const int i = g % nm, c = g0 + g / nm;
    const int col = c < nleft ? c - nleft : ncols + (c - nleft);
    A[l_to[i] + (long)col * lda] = Lsm[g];
  }
  if (!u12) {
    cluster_wait();
    return;
  }
  __syncwarp();
  cluster_arrive();  // every row is in place
  cluster_wait();
  // U12 = L11^-1 A12 on the right columns' top MN rows, over all the cluster's warps
  panel_u12_solve<T, NB>(MN, ncols, nright, crank * (PT / 32) + warp, C * (PT / 32), A, lda);
}

// Fallback for panels taller than a cluster can hold: one CTA, global memory.
template <typename T>
__global__ void __launch_bounds__(1024)
getf2_global_kernel(int M, int ncols, T *A, long lda, int *ipiv, int roff, int *dinfo) {
  __shared__ T sv[32];
  __shared__ int sp[32];
  __shared__ int piv_row;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int MN = min(M, ncols);
  for (int j = 0; j < MN; j++) {
    T v = T(-1);
    int vp = INT_MAX;
    for (int i = j + tid; i < M; i += blockDim.x) {
      T t = fabs(A[i + (long)j * lda]);
      if (t > v) { v = t; vp = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      T ov = __shfl_xor_sync(0xffffffffu, v, o);
      int op = __shfl_xor_sync(0xffffffffu, vp, o);
      if (ov > v || (ov == v && op < vp)) { v = ov; vp = op; }
    }
    if (lane == 0) { sv[warp] = v; sp[warp] = vp; }
    __syncthreads();
    if (warp == 0) {
      v = lane < (int)(blockDim.x / 32) ? sv[lane] : T(-1);
      vp = lane < (int)(blockDim.x / 32) ? sp[lane] : INT_MAX;
      for (int o = 16; o > 0; o >>= 1) {
        T ov = __shfl_xor_sync(0xffffffffu, v, o);
        int op = __shfl_xor_sync(0xffffffffu, vp, o);
        if (ov > v || (ov == v && op < vp)) { v = ov; vp = op; }
      }
      if (lane == 0) {
        if (v <= T(0)) vp = j;
        piv_row = vp;
        ipiv[j] = roff + vp;
        if (v == T(0)) atomicMin(dinfo, roff + j + 1);
      }
    }
    __syncthreads();
    const int p = piv_row;
    if (p != j)
      for (int k = tid; k < ncols; k += blockDim.x) {
        T t = A[j + (long)k * lda];
        A[j + (long)k * lda] = A[p + (long)k * lda];
        A[p + (long)k * lda] = t;
      }
    __syncthreads();
    const T piv = A[j + (long)j * lda];
    if (piv != T(0)) {
      const bool use_rcp = fabs(piv) >= safmin<T>();
      const T rcp = T(1) / piv;
      for (int i = j + 1 + tid; i < M; i += blockDim.x) {
        T l = use_rcp ? A[i + (long)j * lda] * rcp : A[i + (long)j * lda] / piv;
        A[i + (long)j * lda] = l;
        for (int k = j + 1; k < ncols; k++) A[i + (long)k * lda] -= l * A[j + (long)k * lda];
      }
    }
    __syncthreads();
  }
}

int g_max_cluster = 0;

template <typename T, int NB, int RPT>
bool launch_cluster_panel(int M, int ncols, T *A, long lda, int *ipiv, int roff, int *dinfo,
                          cudaStream_t st) {
  int C = cdiv(M, PT * RPT);
  if (C > g_max_cluster) return false;
  auto kern = getf2_cluster_kernel<T, NB, RPT>;
  static bool configured = false;
  if (!configured) {
    ATLB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    configured = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(PT, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATLB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, M, ncols, A, lda, ipiv, roff, dinfo));
  return true;
}

void init_max_cluster() {
  if (g_max_cluster) return;
  // largest cluster of PT-thread CTAs the device can co-schedule (16 needs
  // the non-portable opt-in; fall back to the portable 8)
  auto kern = getf2_cluster_kernel<double, 32, 1>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16, 1, 1);
  cfg.blockDim = dim3(PT, 1, 1);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
  if (e != cudaSuccess) { cudaGetLastError(); n = 0; }
  g_max_cluster = n > 0 ? 16 : 8;
}

template <typename T>
constexpr int fused_smem_bytes() { return 32 * PT * (int)sizeof(T); }

// Largest cluster of the fused panel kernel (<= 16 CTAs, ~140 KB shared
// memory each) the device can co-schedule; 0 when none.
template <typename T>
int max_cluster_fused() {
  static int cached = -1;
  if (cached >= 0) return cached;
  auto kern = getf2_fused_kernel<T, 32>;
  cached = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, fused_smem_bytes<T>()) !=
          cudaSuccess) {
    cudaGetLastError();
    return cached;
  }
  for (int c : {kMaxPanelCluster, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c, 1, 1);
    cfg.blockDim = dim3(PT, 1, 1);
    cfg.dynamicSmemBytes = fused_smem_bytes<T>();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) { cudaGetLastError(); n = 0; }
    if (n > 0) { cached = c; break; }
  }
  return cached;
}

// Factor the M x ncols panel at A (rows 0.., ipiv + roff numbering) and, when
// nleft / nright > 0, interchange the rows of the block columns beside it and
// solve its right columns' top rows (see getf2_fused_kernel).
template <typename T>
bool launch_fused_panel(int M, int ncols, T *A, long lda, int *ipiv, int roff, int *dinfo, int nleft,
                        int nright, cudaStream_t st) {
  if (ncols > 32 || nleft + nright > 256) return false;  // the interchange staging holds 64 x 256
  const int C = cdiv(M, PT);
  if (C > max_cluster_fused<T>()) return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(PT, 1, 1);
  cfg.dynamicSmemBytes = fused_smem_bytes<T>();
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATLB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, getf2_fused_kernel<T, 32>, M, ncols, A, lda, ipiv, roff, dinfo,
                                     nleft, nright));
  return true;
}

bool fused_panel_disabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("ATLAS_B200_PANEL");
    v = (e && strcmp(e, "cluster") == 0) ? 1 : 0;
  }
  return v == 1;
}

// Panel width the cluster kernel supports for M rows.
int panel_nb(int M) {
  init_max_cluster();
  if (M <= g_max_cluster * PT) return 32;
  if (M <= g_max_cluster * PT * 2) return 16;
  if (M <= g_max_cluster * PT * 4) return 8;
  return 8;
}

template <typename T>
void panel(int M, int ncols, T *A, long lda, int *ipiv, int roff, int *dinfo, cudaStream_t st) {
  bool ok = !fused_panel_disabled() && launch_fused_panel<T>(M, ncols, A, lda, ipiv, roff, dinfo, 0, 0, st);
  if (ok) return;
  if (ncols <= 32 && M <= g_max_cluster * PT) ok = launch_cluster_panel<T, 32, 1>(M, ncols, A, lda, ipiv, roff, dinfo, st);
  else if (ncols <= 16 && M <= g_max_cluster * PT * 2) ok = launch_cluster_panel<T, 16, 2>(M, ncols, A, lda, ipiv, roff, dinfo, st);
  else if (ncols <= 8 && M <= g_max_cluster * PT * 4) ok = launch_cluster_panel<T, 8, 4>(M, ncols, A, lda, ipiv, roff, dinfo, st);
  if (!ok) {
    getf2_global_kernel<T><<<1, 1024, 0, st>>>(M, ncols, A, lda, ipiv, roff, dinfo);
    ATLB_CUDA_CHECK(cudaGetLastError());
  }
}

// trailing update A22 -= A21 * A12 (FP64 DMMA, or the FP32 GEMM supplied)
void update_gemm(SgemmFn, int M, int N, int K, const double *A21, const double *A12, double *A22,
                 long lda, cudaStream_t st) {
  dgemm_dev(kNoTrans, kNoTrans, M, N, K, -1.0, A21, lda, A12, lda, 1.0, A22, lda, st);
}
void update_gemm(SgemmFn fn, int M, int N, int K, const float *A21, const float *A12, float *A22,
                 long lda, cudaStream_t st) {
  (fn ? fn : sgemm_dev)(kNoTrans, kNoTrans, M, N, K, -1.f, A21, lda, A12, lda, 1.f, A22, lda, st, 0);
}

template <typename T>
void getrf_rec(int off, int M, int N, T *A, long lda, int *ipiv, int *dinfo, cudaStream_t st,
               SgemmFn gemm) {
  const int MN = std::min(M, N);
  if (MN <= 0) return;
  T *Ad = A + off + (long)off * lda;  // diagonal block start
  const int nb = panel_nb(M);
  if (MN <= nb) {
    panel<T>(M, MN, Ad, lda, ipiv + off, off, dinfo, st);
    if (N > MN) {
      laswp_dev<T>(N - MN, A + (long)(off + MN) * lda, lda, off, off + MN, ipiv, 1, st);
      trsm_dev<T>(kLeft, kLower, kNoTrans, kUnit, MN, N - MN, T(1), Ad, lda,
                  Ad + (long)MN * lda, lda, st, gemm);
    }
    return;
  }
  const int Nl = std::max(nb, (MN / 2) / nb * nb), Nr = N - Nl;
  getrf_rec<T>(off, M, Nl, A, lda, ipiv, dinfo, st, gemm);
  laswp_dev<T>(Nr, A + (long)(off + Nl) * lda, lda, off, off + Nl, ipiv, 1, st);
  T *A12 = Ad + (long)Nl * lda;
  trsm_dev<T>(kLeft, kLower, kNoTrans, kUnit, Nl, Nr, T(1), Ad, lda, A12, lda, st, gemm);
  T *A21 = Ad + Nl, *A22 = A12 + Nl;
  update_gemm(gemm, M - Nl, Nr, Nl, A21, A12, A22, lda, st);
  getrf_rec<T>(off + Nl, M - Nl, Nr, A, lda, ipiv, dinfo, st, gemm);
  laswp_dev<T>(Nl, A + (long)off * lda, lda, off + Nl, off + MN, ipiv, 1, st);
}

// C (m x nr) -= A (m x k) * B (k x nr), k <= 32, nr <= 256, one leading
// dimension: the update of a block column's remaining columns by one leaf
// panel.  Small and skinny, so a plain GEMM pays its K-loop pipeline and
// tiling for a single 32-deep step.  Here a CTA takes a 64 x 64 tile of C
// (two CTAs per SM, the grid covering m x nr): it copies its 64-row slice of
// A and 64-column slice of B into shared memory (cp.async, every copy in
// flight at once) while its threads load their old C values into registers,
// so it waits for memory once; every thread then computes RU_RT rows (16
// apart, so a half-warp touches 16 consecutive rows of a column) x RU_CQ
// columns (16 apart).  Measured at order 8192 (FP32): 64 x 64 tiles take
// about half the time of 32-row x all-column tiles at one CTA per SM.
constexpr int RU_RT = 4, RU_CQ = 4, RU_BR = 16 * RU_RT, RU_BC = 16 * RU_CQ;

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool pred) {
  if (sizeof(T) == 8) cp_async8(dst, src, pred);
  else cp_async4(dst, src, pred);
}

template <typename T>
__global__ void __launch_bounds__(256, 2)
rank_update_kernel(int m, int nr, int k, const T *__restrict__ A, const T *__restrict__ B, T *__restrict__ C,
                   long lda) {
  __shared__ __align__(16) T sA[32][RU_BR];
  __shared__ __align__(16) T sB[32][RU_BC + 1];
  const int tid = threadIdx.x, r0 = blockIdx.x * RU_BR, c0 = blockIdx.y * RU_BC;
  const int ncl = min(RU_BC, nr - c0);
  const int tr = tid % 16, tc = tid / 16;  // rows r0 + tr + 16 a, columns c0 + tc + 16 q
#pragma unroll
  for (int e = 0; e < 32 * RU_BR / 256; e++) {
    const int idx = tid + 256 * e, r = idx % RU_BR, i = idx / RU_BR;
    const bool ok = i < k && r0 + r < m;
    cp_async_elem(&sA[i][r], ok ? A + r0 + r + (long)i * lda : A, ok);
  }
#pragma unroll
  for (int e = 0; e < 32 * RU_BC / 256; e++) {
    const int idx = tid + 256 * e, i = idx % 32, c = idx / 32;
    const bool ok = i < k && c < ncl;
    cp_async_elem(&sB[i][c], ok ? B + i + (long)(c0 + c) * lda : B, ok);
  }
  cp_async_commit();
  T old[RU_RT][RU_CQ];
#pragma unroll
  for (int q = 0; q < RU_CQ; q++)
#pragma unroll
    for (int a = 0; a < RU_RT; a++) {
      const int r = r0 + tr + 16 * a, c = tc + 16 * q;
      old[a][q] = (c < ncl && r < m) ? C[r + (long)(c0 + c) * lda] : T(0);
    }
  cp_async_wait<0>();
  __syncthreads();
  T acc[RU_RT][RU_CQ];
#pragma unroll
  for (int a = 0; a < RU_RT; a++)
#pragma unroll
    for (int q = 0; q < RU_CQ; q++) acc[a][q] = T(0);
#pragma unroll 8
  for (int i = 0; i < 32; i++) {
    T av[RU_RT], bv[RU_CQ];
#pragma unroll
    for (int a = 0; a < RU_RT; a++) av[a] = sA[i][tr + 16 * a];
#pragma unroll
    for (int q = 0; q < RU_CQ; q++) bv[q] = sB[i][tc + 16 * q];
#pragma unroll
    for (int a = 0; a < RU_RT; a++)
#pragma unroll
      for (int q = 0; q < RU_CQ; q++) acc[a][q] = fma(av[a], bv[q], acc[a][q]);
  }
#pragma unroll
  for (int q = 0; q < RU_CQ; q++)
#pragma unroll
    for (int a = 0; a < RU_RT; a++) {
      const int r = r0 + tr + 16 * a, c = tc + 16 * q;
      if (c < ncl && r < m) C[r + (long)(c0 + c) * lda] = old[a][q] - acc[a][q];
    }
}

template <typename T>
void rank_update(int m, int nr, int k, const T *A, const T *B, T *C, long lda, cudaStream_t st) {
  rank_update_kernel<T><<<dim3(cdiv(m, RU_BR), cdiv(nr, RU_BC)), 256, 0, st>>>(m, nr, k, A, B, C, lda);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// Block column [j, j + jb) of the factorization, rows j..M-1, as 32-column
// leaves: each leaf is one fused panel launch (factor + interchanges across
// the block + U12 solve) followed by one GEMM updating the block's columns
// right of the leaf.  The pivots are those of the reference's recursion
// (partial pivoting does not depend on the blocking).  Returns false when
// the rows do not fit one cluster (the caller then uses the recursion).
template <typename T>
bool getrf_block(int j, int M, int jb, T *A, long lda, int *ipiv, int *dinfo, cudaStream_t st,
                 SgemmFn gemm) {
  if (fused_panel_disabled() || cdiv(M - j, PT) > max_cluster_fused<T>()) return false;
  for (int l = 0; l < jb; l += 32) {
    const int c = j + l, w = std::min(32, jb - l), m = M - c;
    if (m <= 0) break;
    const int nright = jb - l - w;
    T *Ac = A + c + (long)c * lda;
    launch_fused_panel<T>(m, w, Ac, lda, ipiv + c, c, dinfo, l, nright, st);
    if (nright > 0 && m - w > 0)  // rank-w update of the block's columns right of the leaf
      rank_update<T>(m - w, nright, w, Ac + w, Ac + (long)w * lda, Ac + w + (long)w * lda, lda, st);
  }
  return true;
}

}  // namespace

bool lookahead_enabled() { return tune(kTuneLookahead) != 0; }

// Outer loop: NBO-column block panels (NBO tunable, 256 by default), each factored by the recursion above
// (restricted to the panel's columns); the panel's row interchanges are then
// applied to the columns on both sides and the trailing matrix is updated with
// one TRSM and one large GEMM (the reference's recursion would issue the same
// updates as a cascade of smaller ones; the pivots are the same).
template <typename T>
void getrf_dev(int M, int N, T *A, long lda, int *ipiv, int *dinfo, cudaStream_t st,
               SgemmFn gemm) {
  // the launch sequence depends only on (M, N, lda, pointers): replayed as a graph
  // multiple of 32, <= 256 (the fused panel's limit); the FP32 factorization has its own
  const int NBO = tune(sizeof(T) == 4 ? kTuneSgetrfNB : kTuneGetrfNB);
  const std::vector<unsigned long long> key = {1ull + sizeof(T), (unsigned long long)tune_generation(),
      (unsigned long long)M,
      (unsigned long long)N, (unsigned long long)lda, (unsigned long long)(uintptr_t)A,
      (unsigned long long)(uintptr_t)ipiv, (unsigned long long)(uintptr_t)dinfo,
      (unsigned long long)(uintptr_t)gemm, (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    set_info_kernel_launch(dinfo, st);
    const int MN = std::min(M, N), nblk = cdiv(MN, NBO);
    if (nblk <= 1 || !lookahead_enabled()) {
      for (int j = 0; j < MN; j += NBO) {
        const int jb = std::min(NBO, MN - j);
        T *Ad = A + j + (long)j * lda;
        if (!getrf_block<T>(j, M, jb, A, lda, ipiv, dinfo, st, gemm))   // panel: rows j.., columns j..j+jb
          getrf_rec<T>(j, M - j, jb, A, lda, ipiv, dinfo, st, gemm);
        if (j > 0) laswp_dev<T>(j, A, lda, j, j + jb, ipiv, 1, st);  // left of the panel
        const int nr = N - j - jb;
        if (nr > 0) {
          T *A12 = Ad + (long)jb * lda;
          laswp_dev<T>(nr, A + (long)(j + jb) * lda, lda, j, j + jb, ipiv, 1, st);
          trsm_llu_small_dev<T>(jb, nr, Ad, lda, A12, lda, st);
          if (M - j - jb > 0) update_gemm(gemm, M - j - jb, nr, jb, Ad + jb, A12, A12 + jb, lda, st);
        }
      }
    } else {
      // Look-ahead of depth one: while the main stream applies block k to
      // the trailing matrix, the side stream (higher priority) first applies
      // block k to the next block column only and then factors it, so the
      // latency-bound panel runs under the bandwidth/tensor-bound update.
      // Writes of the two streams never overlap: the side stream owns the
      // next block column, the main stream everything to its right and the
      // interchanges on the left.
      cudaStream_t s1 = side_stream();
      if (!getrf_block<T>(0, M, std::min(NBO, MN), A, lda, ipiv, dinfo, st, gemm))
        getrf_rec<T>(0, M, std::min(NBO, MN), A, lda, ipiv, dinfo, st, gemm);
      for (int k = 0; k < nblk; k++) {
        const int j = k * NBO, jb = std::min(NBO, MN - j), jn = j + jb;
        const int jbn = k + 1 < nblk ? std::min(NBO, MN - jn) : 0;
        T *Ad = A + j + (long)j * lda;
        if (k > 0) ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, side_event(2 + (k & 1)), 0));  // block k factored
        if (jbn > 0) {
          ATLB_CUDA_CHECK(cudaEventRecord(side_event(k & 1), st));  // updates by blocks < k are in
          ATLB_CUDA_CHECK(cudaStreamWaitEvent(s1, side_event(k & 1), 0));
          SideScope side;
          T *An = A + (long)jn * lda;
          laswp_dev<T>(jbn, An, lda, j, jn, ipiv, 1, s1);
          trsm_llu_small_dev<T>(jb, jbn, Ad, lda, An + j, lda, s1);
          if (M - jn > 0) update_gemm(gemm, M - jn, jbn, jb, Ad + jb, An + j, An + jn, lda, s1);
          if (!getrf_block<T>(jn, M, jbn, A, lda, ipiv, dinfo, s1, gemm))
            getrf_rec<T>(jn, M - jn, jbn, A, lda, ipiv, dinfo, s1, gemm);
          ATLB_CUDA_CHECK(cudaEventRecord(side_event(2 + ((k + 1) & 1)), s1));
        }
        if (j > 0) laswp_dev<T>(j, A, lda, j, jn, ipiv, 1, st);
        const int c0 = jn + jbn, nr = N - c0;
        if (nr > 0) {
          T *Ar = A + (long)c0 * lda;
          laswp_dev<T>(nr, Ar, lda, j, jn, ipiv, 1, st);
          trsm_llu_small_dev<T>(jb, nr, Ad, lda, Ar + j, lda, st);
          // the trailing update may leave SMs to the side stream's panel
          const int reserve = jbn > 0 ? tune(kTuneLookaheadReserve) : 0;
          GemmCtaCap cap(reserve > 0 ? std::max(1, num_sms() - reserve) : 0);
          if (M - jn > 0) update_gemm(gemm, M - jn, nr, jb, Ad + jb, Ar + j, Ar + jn, lda, st);
        }
      }
    }
    finish_info_kernel_launch(dinfo, st);
  });
}
template void getrf_dev<double>(int, int, double *, long, int *, int *, cudaStream_t, SgemmFn);
template void getrf_dev<float>(int, int, float *, long, int *, int *, cudaStream_t, SgemmFn);

template <typename T>
void getrs_dev(int trans, int N, int NRHS, const T *A, long lda, const int *ipiv, T *B, long ldb,
               cudaStream_t st, SgemmFn gemm) {
  // ATL_getrs column-major (src/lapack/ATL_getrs.c:34-50)
  if (N <= 0 || NRHS <= 0) return;
  if (NRHS <= kTrsvMaxRhs) {  // few right-hand sides: blocked solves, one launch per 8 columns
    if (trans == kNoTrans) {
      laswp_dev<T>(NRHS, B, ldb, 0, N, ipiv, 1, st);
      trsv_dev<T>(kLower, kNoTrans, kUnit, N, NRHS, A, lda, B, ldb, st);
      trsv_dev<T>(kUpper, kNoTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
    } else {
      trsv_dev<T>(kUpper, kTrans, kNonUnit, N, NRHS, A, lda, B, ldb, st);
      trsv_dev<T>(kLower, kTrans, kUnit, N, NRHS, A, lda, B, ldb, st);
      laswp_dev<T>(NRHS, B, ldb, 0, N, ipiv, -1, st);
    }
    return;
  }
  if (trans == kNoTrans) {
    laswp_dev<T>(NRHS, B, ldb, 0, N, ipiv, 1, st);
    trsm_dev<T>(kLeft, kLower, kNoTrans, kUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
    trsm_dev<T>(kLeft, kUpper, kNoTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
  } else {
    trsm_dev<T>(kLeft, kUpper, kTrans, kNonUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
    trsm_dev<T>(kLeft, kLower, kTrans, kUnit, N, NRHS, T(1), A, lda, B, ldb, st, gemm);
    laswp_dev<T>(NRHS, B, ldb, 0, N, ipiv, -1, st);
  }
}
template void getrs_dev<double>(int, int, int, const double *, long, const int *, double *, long,
                                cudaStream_t, SgemmFn);
template void getrs_dev<float>(int, int, int, const float *, long, const int *, float *, long,
                               cudaStream_t, SgemmFn);

}  // namespace atlb

// ---------------------------------------------------------------------------
// LU without pivoting, used by the mixed-precision solver after a random
// butterfly transformation has made pivoting unnecessary (rbt.cu).  Blocked
// right-looking: each NBD x NBD diagonal block is factored by one CTA in
// shared memory, the block column below it and the block row right of it by
// TRSM, and the trailing matrix by one GEMM.  A zero pivot lowers *dinfo.
namespace atlb {
namespace {

constexpr int NBD = 128;

// LU without pivoting of one NBD x NBD diagonal block, one CTA: thread
// (i, g) keeps row i's columns g, g+4, ... in registers.  Each step needs
// the pivot row and the pivot column; the threads that finish them in step
// j-1 publish them to a double-buffered shared copy, so a step costs one
// barrier.
template <typename T>
__global__ void __launch_bounds__(512)
lu_nopiv_diag_kernel(int n, T *A, long lda, int *dinfo, int ioff) {
  static_assert(NBD == 128, "4 threads per row, 32 columns each");
  __shared__ T prow[2][NBD];
  __shared__ T pcol[2][NBD];
  const int tid = threadIdx.x, i = tid % NBD, g = tid / NBD;
  T a[NBD / 4];
  const long step4 = 4 * lda;
  {
    const T *src = A + (i < n ? i : 0) + (long)g * lda;
#pragma unroll
    for (int m = 0; m < NBD / 4; m++) {
      a[m] = (i < n && g + 4 * m < n) ? src[0] : T(0);
      src += (g + 4 * m + 4 < n) ? step4 : 0;
    }
  }
  if (i == 0) {
#pragma unroll
    for (int m = 0; m < NBD / 4; m++) prow[0][g + 4 * m] = a[m];
  }
  if (g == 0) pcol[0][i] = a[0];
  __syncthreads();
#pragma unroll 1
  for (int j = 0; j < n; j++) {
    const int b = j & 1;
    const T p = prow[b][j];
    if (p == T(0)) {
      if (tid == 0) atomicMin(dinfo, ioff + j + 1);
      break;  // uniform: every thread read the same pivot
    }
    if (i > j && i < n) {
      const T l = pcol[b][i] * (T(1) / p);
#pragma unroll
      for (int m = 0; m < NBD / 4; m++) {
        const int k = g + 4 * m;
        if (k == j) a[m] = l;
        else if (k > j) a[m] = fma(-l, prow[b][k], a[m]);
      }
    }
    if (i == j + 1) {
#pragma unroll
      for (int m = 0; m < NBD / 4; m++) prow[b ^ 1][g + 4 * m] = a[m];
    }
    if (g == ((j + 1) & 3) && i > j) {
      T v = T(0);
#pragma unroll
      for (int m = 0; m < NBD / 4; m++)
        if (g + 4 * m == j + 1) v = a[m];
      pcol[b ^ 1][i] = v;
    }
    __syncthreads();
  }
  if (i < n) {
    T *dst = A + i + (long)g * lda;
#pragma unroll
    for (int m = 0; m < NBD / 4; m++) {
      if (g + 4 * m < n) dst[0] = a[m];
      dst += step4;
    }
  }
}

}  // namespace

template <typename T>
void getrf_nopiv_dev(int N, T *A, long lda, int *dinfo, cudaStream_t st, SgemmFn gemm) {
  const std::vector<unsigned long long> key = {11ull + sizeof(T), (unsigned long long)N,
      (unsigned long long)lda, (unsigned long long)(uintptr_t)A, (unsigned long long)(uintptr_t)dinfo,
      (unsigned long long)(uintptr_t)gemm, (unsigned long long)(uintptr_t)st};
  run_graph(key, st, [&]() {
    set_info_kernel_launch(dinfo, st);
    for (int j = 0; j < N; j += NBD) {
      const int jb = std::min(NBD, N - j), nr = N - j - jb;
      T *Ad = A + j + (long)j * lda;
      lu_nopiv_diag_kernel<T><<<1, 512, 0, st>>>(jb, Ad, lda, dinfo, j);
      ATLB_CUDA_CHECK(cudaGetLastError());
      if (nr <= 0) break;
      T *A21 = Ad + jb, *A12 = Ad + (long)jb * lda;
      trsm_dev<T>(kRight, kUpper, kNoTrans, kNonUnit, nr, jb, T(1), Ad, lda, A21, lda, st, gemm);
      trsm_dev<T>(kLeft, kLower, kNoTrans, kUnit, jb, nr, T(1), Ad, lda, A12, lda, st, gemm);
      update_gemm(gemm, nr, nr, jb, A21, A12, A12 + jb, lda, st);
    }
    finish_info_kernel_launch(dinfo, st);
  });
}
template void getrf_nopiv_dev<double>(int, double *, long, int *, cudaStream_t, SgemmFn);
template void getrf_nopiv_dev<float>(int, float *, long, int *, cudaStream_t, SgemmFn);

}  // namespace atlb
