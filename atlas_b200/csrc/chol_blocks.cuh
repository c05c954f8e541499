// Blocked Cholesky building blocks in shared memory, for one CTA of 256
// threads: the batched solver (batched.cu) factors whole small matrices with
// them, the blocked potrf (chol.cu) its diagonal blocks.
#pragma once
#include <cuda_runtime.h>

namespace atlb {
namespace cholb {

// C (rows < mt, columns < nc <= mt, lower part i >= k) -= P P^T, P = mt x jb
// (ld lds, shared memory); C in shared or global memory (ldc).  16 x 16
// threads, 4 x 4 register tiles over 64 x 64 blocks of the lower trapezoid.
template <typename T, typename CT>
__device__ __forceinline__ void syrk_lower_update(int mt, int nc, int jb, const T *P, int lds, CT *C, long ldc) {
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  for (int ib = 0; ib < mt; ib += 64)
    for (int kb = 0; kb <= ib && kb < nc; kb += 64) {
      T acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = T(0);
      for (int q = 0; q < jb; q++) {
        T pi[4], pk[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const int i = ib + tx + 16 * a;
          pi[a] = i < mt ? P[i + q * lds] : T(0);
        }
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int k = kb + ty + 16 * b;
          pk[b] = k < nc ? P[k + q * lds] : T(0);
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) acc[a][b] = fma(pi[a], pk[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int i = ib + tx + 16 * a, k = kb + ty + 16 * b;
          if (i < mt && k < nc && k <= i) C[i + (long)k * ldc] -= acc[a][b];
        }
    }
}

// Leading dimension for an order-n matrix in shared memory: the smallest
// value >= n that is 8 (mod 16) doubles, so that the 8 x 4 operand fragments
// of the FP64 MMA below (lanes: 8 rows x 4 columns) fall in distinct banks.
__host__ __device__ constexpr int ld_for(int n) { return (n + 7) / 16 * 16 + 8; }

// d += a b on one m8n8k4 FP64 tensor-core tile (PTX mma.m8n8k4 .f64
// fragments: a = A[g][t], b = B[t][g], d = D[g][2t..2t+1], g = lane / 4,
// t = lane % 4)
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// FP64 form of syrk_lower_update on the tensor cores: each warp of the 256
// owns a 16 x 32 part of every 64 x 64 block (2 x 4 tiles of 8 x 8), skips
// the tiles strictly above the diagonal, starts its accumulators from C and
// adds (-P) P^T in k-steps of 4 (P read as zero beyond jb); KJ > 0 fixes jb
// at compile time.
template <int KJ, typename CT>
__device__ __forceinline__ void syrk_lower_update_dmma(int mt, int nc, int jb_, const double *P, int lds, CT *C,
                                                       long ldc) {
  const int jb = KJ ? KJ : jb_;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
  for (int ib = 0; ib < mt; ib += 64)
    for (int kb = 0; kb <= ib && kb < nc; kb += 64) {
      const int r0 = ib + wr, c0 = kb + wc;
      if (r0 >= mt || c0 >= nc || c0 > r0 + 15) continue;  // warp-uniform: nothing of this warp's part is stored
      double acc[2][4][2];
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int i = r0 + 8 * a + g, k = c0 + 8 * b + 2 * t + e;
            acc[a][b][e] = (i < mt && k < nc && k <= i) ? double(C[i + (long)k * ldc]) : 0.0;
          }
#pragma unroll 4
      for (int q = 0; q < jb; q += 4) {
        const int qq = q + t;
        double av[2], bv[4];
#pragma unroll
        for (int a = 0; a < 2; a++) {
          const int i = r0 + 8 * a + g;
          av[a] = (i < mt && qq < jb) ? -P[i + qq * lds] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int k = c0 + 8 * b + g;
          bv[b] = (k < nc && qq < jb) ? P[k + qq * lds] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int b = 0; b < 4; b++)
            if (c0 + 8 * b <= r0 + 8 * a + 7) dmma_8x8x4(acc[a][b], av[a], bv[b]);
      }
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int i = r0 + 8 * a + g, k = c0 + 8 * b + 2 * t + e;
            if (i < mt && k < nc && k <= i) C[i + (long)k * ldc] = acc[a][b][e];
          }
    }
}

// the trailing update of a 16-column panel: FP64 on the tensor cores, FP32 on the FMA pipes
template <typename T, typename CT>
__device__ __forceinline__ void syrk_panel(int mt, int nc, int jb, const T *P, int lds, CT *C, long ldc) {
  if constexpr (sizeof(T) == 8) {
    if (jb == 16) syrk_lower_update_dmma<16>(mt, nc, jb, P, lds, C, ldc);
    else syrk_lower_update_dmma<0>(mt, nc, jb, P, lds, C, ldc);
  } else {
    syrk_lower_update(mt, nc, jb, P, lds, C, ldc);
  }
}

// Cholesky of the jb <= 16 columns of the m x jb panel at s (ld lds, rows
// from the panel's diagonal).  Warp 0 factors the jb x jb diagonal block:
// lane i holds row i in registers and every lane keeps its own copy of the
// jb diagonal entries, so the column-to-column chain (diagonal -> 1/sqrt ->
// multipliers -> next diagonal) has no shuffle and no block barrier; each
// finished column goes to shared memory, where the lanes read the
// multipliers back after a warp barrier.  Then every thread solves rows of
// L21 = A21 L11^-T on its own.  Right-looking order within each row, as the
// unblocked algorithm: column c is scaled by 1/sqrt(d_c), then its multiple
// is subtracted from columns c+1.. .  JB > 0 fixes jb at compile time.
// Returns 0 or the first non-positive pivot (1-based, panel-relative), the
// same in every thread; the columns before it are then factored and stored,
// the rest of the panel is not.
template <typename T, int JB>
__device__ int chol_panel_w(T *s, int lds, int m, int jb_) {
  __shared__ T s_rinv[16];
  __shared__ int s_fail;
  const int jb = JB ? JB : jb_;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid < 32) {
    const int i = tid;
    T r[16], dd[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      r[k] = (i < jb && k < jb && k <= i) ? s[i + k * lds] : T(0);
      dd[k] = k < jb ? s[k + k * lds] : T(1);
    }
    int fail = 0;
#pragma unroll
    for (int c = 0; c < 16; c++) {
      if (c >= jb) continue;
      const T d = dd[c];
      if (!(d > T(0)) && !fail) fail = c + 1;  // later columns run on, unstored
      const T ri = rsqrt(d);
      const T l = (i == c ? d : r[c]) * ri;  // L[i][c] (zero above the diagonal)
      if (!fail && i >= c && i < jb) s[i + c * lds] = l;
      if (i == 0) s_rinv[c] = ri;
      __syncwarp();
#pragma unroll
      for (int k = c + 1; k < 16; k++) {
        if (k >= jb) continue;
        const T lk = fail ? T(0) : s[k + c * lds];
        dd[k] = fma(-lk, lk, dd[k]);
        if (i >= k) r[k] = fma(-l, lk, r[k]);
      }
    }
    if (i == 0) s_fail = fail;
  }
  __syncthreads();
  const int fail = s_fail;
  if (fail) {
    __syncthreads();  // s_fail read by all before a later call rewrites it
    return fail;
  }
  for (int i = jb + tid; i < m; i += nt) {
    T x[16];
#pragma unroll
    for (int c = 0; c < 16; c++) x[c] = c < jb ? s[i + c * lds] : T(0);
#pragma unroll
    for (int c = 0; c < 16; c++) {
      if (c >= jb) continue;
      x[c] = x[c] * s_rinv[c];
#pragma unroll
      for (int k = c + 1; k < 16; k++)
        if (k < jb) x[k] = fma(-x[c], s[k + c * lds], x[k]);
    }
#pragma unroll
    for (int c = 0; c < 16; c++)
      if (c < jb) s[i + c * lds] = x[c];
  }
  __syncthreads();
  return 0;
}

template <typename T>
__device__ int chol_panel16(T *s, int lds, int m, int jb) {
  return jb == 16 ? chol_panel_w<T, 16>(s, lds, m, jb) : chol_panel_w<T, 0>(s, lds, m, jb);
}

// Cholesky of the jb columns of the m x jb panel at s (ld lds, rows from the
// panel's diagonal): 16-column sub-panels, each followed by the update of the
// panel's columns right of it (a lower trapezoid).  Returns 0 or the first
// non-positive pivot (1-based, panel-relative), the same in every thread; on
// failure the panel is left partly factored.
template <typename T>
__device__ int chol_panel(T *s, int lds, int m, int jb) {
  for (int j = 0; j < jb; j += 16) {
    const int w = min(16, jb - j), rest = jb - j - w;
    T *P = s + j + j * lds;
    const int f = chol_panel16(P, lds, m - j, w);
    if (f) return j + f;
    if (rest > 0) {
      syrk_panel(m - j - w, rest, w, P + w, lds, P + w + w * lds, lds);
      __syncthreads();
    }
  }
  return 0;
}

// blocked right-looking Cholesky of an n x n lower matrix in shared memory
// (ld lds); returns 0 or the first non-positive pivot (1-based), the matrix
// then partly factored
template <typename T>
__device__ int chol_smem(T *s, int lds, int n) {
  return chol_panel(s, lds, n, n);
}

}  // namespace cholb
}  // namespace atlb
