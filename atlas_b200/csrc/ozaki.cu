// Split-integer ("Ozaki") DGEMM on the INT8 tensor cores.  No counterpart in
// the reference (ATLAS's DGEMM is plain FP64).
//
// Each row i of op(A) is scaled by 2^-e_i (e_i = exponent of its largest
// magnitude, so the scaled row lies in (-1, 1)) and each column j of op(B) by
// 2^-f_j.  A scaled value v is written as v = 2^-6 * sum_{s=1..S} 2^{-7(s-1)} d_s
// with signed digits d_s in [-64, 64], extracted exactly in FP64 by repeated
// round-to-nearest (every remainder stays in [-1/2, 1/2]).  Then
//
//   C_ij = 2^{e_i + f_j - 12} * sum_{g=2..S+1} 2^{-7(g-2)} * sum_{s+t=g} (A_s B_t)_ij
//
// (terms with s + t > S + 1 are below the last kept digit and dropped).  The
// digit products are exact INT32 sums (|d| <= 64, so K * 64^2 * S stays far
// below 2^31 for K up to 2^20).  The slices are stored row-major as
// [rows][S][Kp] -- A in slice order 1..S, B in reverse order S..1 -- so the
// whole group g is ONE int8 GEMM over the contiguous K-window of width
// (g-1)*Kp: A rows from offset 0, B rows from offset (S-g+1)*Kp.  Each group's
// INT32 result is scaled by powers of two (exact) and accumulated into the
// FP64 C in the GEMM's epilogue, smallest weight first.
#include <algorithm>
#include <cmath>
#include "common.cuh"
#include "kernels.h"
#include "tc_gemm.h"
#include "staging.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

constexpr int MAXS = 12;

// exponent e with max|x| * 2^-e in [1/2, 1) (0 for an all-zero row)
__device__ __forceinline__ int exp_of(double m) { return m > 0.0 ? ilogb(m) + 1 : 0; }

// per-row scale of op(A) (rows x K): rs[i] = 2^e_i
__global__ void row_scale_kernel(int rows, int K, const double *__restrict__ X, long ld, int rcontig,
                                 double *__restrict__ rs, int *__restrict__ re) {
  // rcontig: X(r, k) = X[r + k*ld] (rows contiguous): one thread per row, coalesced
  // otherwise X(r, k) = X[k + r*ld]: one warp per row
  if (rcontig) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double m = 0.0;
    for (int k = 0; k < K; k++) m = fmax(m, fabs(X[r + (long)k * ld]));
    const int e = exp_of(m);
    re[r] = e;
    rs[r] = ldexp(1.0, e);
  } else {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= rows) return;
    double m = 0.0;
    for (int k = lane; k < K; k += 32) m = fmax(m, fabs(X[k + (long)w * ld]));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
      const int e = exp_of(m);
      re[w] = e;
      rs[w] = ldexp(1.0, e);
    }
  }
}

// Slice op(X) (rows x K) into out[r * ldo + pos(s) * Kp + k] with
// pos(s) = s (forward) or S-1-s (reverse); k in [K, Kp) zero-filled.
// 32 x 32 tiles through shared memory so both the FP64 reads and the int8
// writes are coalesced whatever the layout of X.
__global__ void __launch_bounds__(256)
slice_kernel(int rows, int K, int Kp, const double *__restrict__ X, long ld, int rcontig,
             const int *__restrict__ ex, int S, int reverse, signed char *__restrict__ out, long ldo) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int j = ty; j < 32; j += 8) {
    int r, k;
    if (rcontig) { r = r0 + tx; k = k0 + j; } else { k = k0 + tx; r = r0 + j; }
    const double v = (r < rows && k < K) ? X[rcontig ? (r + (long)k * ld) : (k + (long)r * ld)] : 0.0;
    if (rcontig) t[j][tx] = v; else t[tx][j] = v;  // t[k_local][r_local]
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int r = r0 + j, k = k0 + tx;
    if (r < rows && k < Kp) {
      signed char *o = out + (long)r * ldo + k;
      const int e = ex[r];
      double v = t[tx][j];
      double rr = ldexp(v, 6 - e);
      for (int s = 0; s < S; s++) {
        const double q = rint(rr);
        const int pos = reverse ? (S - 1 - s) : s;
        o[(long)pos * Kp] = (signed char)(int)q;
        rr = (rr - q) * 128.0;
      }
    }
  }
}

__global__ void scale_c_kernel(int M, int N, double beta, double *C, long ldc) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    double *p = C + (idx % M) + (idx / M) * ldc;
    *p = beta == 0.0 ? 0.0 : beta * *p;
  }
}

}  // namespace

// C = alpha*op(A)*op(B) + beta*C with S slices (device pointers)
void dgemm_ozaki_dev(int ta, int tb, int M, int N, int K, double alpha, const double *A, long lda,
                     const double *B, long ldb, double beta, double *C, long ldc, int S,
                     cudaStream_t st) {
  if (M <= 0 || N <= 0) return;
  {
    long total = (long)M * N;
    if (beta != 1.0)
      scale_c_kernel<<<(int)std::min<long>((total + 255) / 256, 148L * 16), 256, 0, st>>>(M, N, beta, C, ldc);
  }
  if (K <= 0 || alpha == 0.0) return;
  const int Kp = cdiv(K, 16) * 16;
  const long ldS = (long)S * Kp;
  // workspace: slices of A and B, exponents and scales
  size_t abytes = (size_t)M * ldS, bbytes = (size_t)N * ldS;
  signed char *As = (signed char *)scratch(kSlotOzA, abytes + 256);
  signed char *Bs = (signed char *)scratch(kSlotOzB, bbytes + 256);
  double *sc = (double *)scratch(kSlotOzScale, sizeof(double) * (M + N) + sizeof(int) * (M + N) + 64);
  double *rs = sc, *cs = sc + M;
  int *re = (int *)(sc + M + N), *ce = re + M;
  // op(A)(i,k): rows contiguous when A is not transposed; op(B)^T(j,k) = op(B)(k,j):
  // rows (j) contiguous when B is transposed
  const int a_rc = ta == kNoTrans, b_rc = tb != kNoTrans;
  if (a_rc) row_scale_kernel<<<cdiv(M, 256), 256, 0, st>>>(M, K, A, lda, 1, rs, re);
  else row_scale_kernel<<<cdiv((long)M * 32, 256), 256, 0, st>>>(M, K, A, lda, 0, rs, re);
  if (b_rc) row_scale_kernel<<<cdiv(N, 256), 256, 0, st>>>(N, K, B, ldb, 1, cs, ce);
  else row_scale_kernel<<<cdiv((long)N * 32, 256), 256, 0, st>>>(N, K, B, ldb, 0, cs, ce);
  slice_kernel<<<dim3(cdiv(Kp, 32), cdiv(M, 32)), 256, 0, st>>>(M, K, Kp, A, lda, a_rc, re, S, 0, As, ldS);
  slice_kernel<<<dim3(cdiv(Kp, 32), cdiv(N, 32)), 256, 0, st>>>(N, K, Kp, B, ldb, b_rc, ce, S, 1, Bs, ldS);
  ATLB_CUDA_CHECK(cudaGetLastError());
  tc::EpiParams ep = {};
  ep.Cd = C;
  ep.ldc = ldc;
  ep.rs = rs;
  ep.cs = cs;
  for (int g = S + 1; g >= 2; g--) {  // smallest weight first
    ep.w = alpha * std::ldexp(1.0, -12 - 7 * (g - 2));
    tc::tc_gemm(tc::kKindI8, tc::kEpiF64Acc, As, ldS, Bs + (long)(S - g + 1) * Kp, ldS, M, N,
                (g - 1) * Kp, ep, st);
  }
}

}  // namespace atlb

using namespace atlb;

extern "C" {

int atlb_dgemm_ozaki_dev(int TA, int TB, int M, int N, int K, double alpha, const double *A,
                         int lda, const double *B, int ldb, double beta, double *C, int ldc,
                         int slices) {
  if (TA != kNoTrans && TA != kTrans && TA != kConjTrans) return -1;
  if (TB != kNoTrans && TB != kTrans && TB != kConjTrans) return -2;
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (lda < std::max(1, TA == kNoTrans ? M : K)) return -8;
  if (ldb < std::max(1, TB == kNoTrans ? K : N)) return -10;
  if (ldc < std::max(1, M)) return -13;
  if (slices < 2 || slices > MAXS) return -14;
  dgemm_ozaki_dev(TA == kNoTrans ? kNoTrans : kTrans, TB == kNoTrans ? kNoTrans : kTrans, M, N, K,
                  alpha, A, lda, B, ldb, beta, C, ldc, slices, stream());
  return 0;
}

int atlb_dgemm_ozaki(int TA, int TB, int M, int N, int K, double alpha, const double *A, int lda,
                     const double *B, int ldb, double beta, double *C, int ldc, int slices) {
  if (TA != kNoTrans && TA != kTrans && TA != kConjTrans) return -1;
  if (TB != kNoTrans && TB != kTrans && TB != kConjTrans) return -2;
  if (M < 0) return -3;
  if (N < 0) return -4;
  if (K < 0) return -5;
  if (lda < std::max(1, TA == kNoTrans ? M : K)) return -8;
  if (ldb < std::max(1, TB == kNoTrans ? K : N)) return -10;
  if (ldc < std::max(1, M)) return -13;
  if (slices < 2 || slices > MAXS) return -14;
  if (M == 0 || N == 0) return 0;
  cudaStream_t st = stream();
  const bool tA = TA != kNoTrans, tB = TB != kNoTrans;
  DMat<double> dA = stage_in(kSlotA, A, tA ? K : M, tA ? M : K, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, B, tB ? N : K, tB ? K : N, ldb, true, st);
  DMat<double> dC = stage_in(kSlotC, (const double *)C, M, N, ldc, beta != 0.0, st);
  dgemm_ozaki_dev(tA ? kTrans : kNoTrans, tB ? kTrans : kNoTrans, M, N, K, alpha, dA.d, dA.ld, dB.d,
                  dB.ld, beta, dC.d, dC.ld, slices, st);
  stage_out(C, ldc, dC, M, N, st);
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  return 0;
}

}  // extern "C"
