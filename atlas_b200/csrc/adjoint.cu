// Reverse-mode derivatives (adjoints) of the factorizations and solves.  No
// counterpart in the reference.  All are blocked: every step is a TRMM,
// TRSM or GEMM on the kernels of this library, plus elementwise kernels.
//
//   potrf  A = L L^T (lower):      Abar = (S + S^T)/2,  S = L^-T Phi(L^T Lbar) L^-1,
//                                  Phi = lower triangle with the diagonal halved
//                                  (Murray, "Differentiation of the Cholesky
//                                  decomposition", 2016)
//   potrs  X = A^-1 B:             Bbar = A^-1 Xbar,  Abar -= (Bbar X^T + X Bbar^T)/2
//   getrs  X = A^-1 B:             Bbar = A^-T Xbar,  Abar -= Bbar X^T
//   getrf  A = P L U (unit L):     Abar = P L^-T (stril(L^T Lbar) + triu(Ubar U^T)) U^-T
//
// The symmetric adjoints (potrf, potrs) are returned as full symmetric
// matrices: the gradient with respect to a symmetric A.
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

enum { kPartLower = 0, kPartStrictLower = 1, kPartUpper = 2, kPartPhi = 3 };

// D = the selected part of S (zero elsewhere); elementwise, so D may be S
__global__ void part_kernel(int n, const double *S, long lds, double *D, long ldd, int mode) {
  long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    const double v = S[i + (long)j * lds];
    double o;
    switch (mode) {
      case kPartLower: o = i >= j ? v : 0.0; break;
      case kPartStrictLower: o = i > j ? v : 0.0; break;
      case kPartUpper: o = i <= j ? v : 0.0; break;
      default: o = i > j ? v : (i == j ? 0.5 * v : 0.0); break;
    }
    D[i + (long)j * ldd] = o;
  }
}

// D = (S + S^T)/2 (D must not alias S)
__global__ void symmetrize_avg_kernel(int n, const double *S, long lds, double *D, long ldd) {
  long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    D[i + (long)j * ldd] = 0.5 * (S[i + (long)j * lds] + S[j + (long)i * lds]);
  }
}

// D = X + Y
__global__ void add_kernel(int n, const double *X, long ldx, const double *Y, long ldy, double *D, long ldd) {
  long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), j = (int)(idx / n);
    D[i + (long)j * ldd] = X[i + (long)j * ldx] + Y[i + (long)j * ldy];
  }
}

__global__ void copy_kernel(int m, int n, const double *S, long lds, double *D, long ldd) {
  long total = (long)m * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % m), j = (int)(idx / m);
    D[i + (long)j * ldd] = S[i + (long)j * lds];
  }
}

inline int gfor(long total) { return (int)std::min<long>((total + 255) / 256, 148L * 16); }

// ---------------------------------------------------------------- batched
// One persistent launch for many small problems (order <= kAdjMaxN): each CTA
// takes problems in turn and works on them in global memory (the per-problem
// working set -- L, the inverse of L, one product -- stays in L2), so no
// shared-memory limit caps the order.
constexpr int kAdjMaxN = 256;
constexpr int AT = 256;  // threads per CTA: a 16 x 16 grid of 4 x 4 output tiles

// X = L^-1 (L lower, non-unit; X lower, ld n): thread t < n solves column t by
// forward substitution, four partial sums to shorten the dependence chain.
__device__ void batched_trinv_lower(int n, const double *L, long ldl, double *X) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    for (int i = 0; i < t; i++) X[i + (long)t * n] = 0.0;
    for (int i = t; i < n; i++) {
      double s0 = (i == t) ? 1.0 : 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int k = t;
      for (; k + 4 <= i; k += 4) {
        s0 -= L[i + (long)k * ldl] * X[k + (long)t * n];
        s1 -= L[i + (long)(k + 1) * ldl] * X[k + 1 + (long)t * n];
        s2 -= L[i + (long)(k + 2) * ldl] * X[k + 2 + (long)t * n];
        s3 -= L[i + (long)(k + 3) * ldl] * X[k + 3 + (long)t * n];
      }
      for (; k < i; k++) s0 -= L[i + (long)k * ldl] * X[k + (long)t * n];
      X[i + (long)t * n] = ((s0 + s1) + (s2 + s3)) / L[i + (long)i * ldl];
    }
  }
}

// C (n x n, ld ldc) = op(A) op(B) over n x n operands, where op(X) = X or X^T
// and only the parts selected by the masks are read: a lower-triangular
// operand (lowA / lowB) has zeros above its diagonal that are not read
// (useful when the stored upper part holds other data).  4 x 4 register tiles.
__device__ void batched_prod(int n, bool ta, bool lowA, const double *A, long lda, bool tb, bool lowB,
                             const double *B, long ldb, double *C, long ldc) {
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  for (int i0 = 0; i0 < n; i0 += 64)
    for (int j0 = 0; j0 < n; j0 += 64) {
      double acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
      for (int k = 0; k < n; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const int i = i0 + tx + 16 * a;  // row of op(A)
          // op(A)(i, k): A(i, k) or A(k, i); lower: zero when the stored row < column
          const int r = ta ? k : i, c = ta ? i : k;
          av[a] = (i < n && (!lowA || r >= c)) ? A[r + (long)c * lda] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int j = j0 + ty + 16 * b;
          const int r = tb ? j : k, c = tb ? k : j;
          bv[b] = (j < n && (!lowB || r >= c)) ? B[r + (long)c * ldb] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const int i = i0 + tx + 16 * a, j = j0 + ty + 16 * b;
          if (i < n && j < n) C[i + (long)j * ldc] = acc[a][b];
        }
    }
}

struct PotrfAdjProb {
  const double *L, *Lbar;
  double *Abar;
  int n, ldl, ldlb, ldab;
};
struct PotrsAdjProb {
  const double *L, *X, *Xbar;
  double *Bbar, *Abar;
  int n, nrhs, ldl, ldx, ldxb, ldbb, ldab;
};

// Abar_p = (S + S^T)/2, S = L^-T Phi(L^T Lbar) L^-1 for every problem p
// (the unbatched atlb_dpotrf_adjoint_dev, one CTA per problem at a time).
// ws: per CTA two n x n buffers (kAdjMaxN^2 each).
__global__ void __launch_bounds__(AT)
potrf_adjoint_batched_kernel(int count, const PotrfAdjProb *__restrict__ P, double *__restrict__ ws) {
  double *X = ws + (size_t)blockIdx.x * 2 * kAdjMaxN * kAdjMaxN;  // L^-1
  double *W = X + (size_t)kAdjMaxN * kAdjMaxN;
  for (int p = blockIdx.x; p < count; p += gridDim.x) {
    const PotrfAdjProb pr = P[p];
    const int n = pr.n;
    if (n <= 0 || n > kAdjMaxN) continue;
    const double *Lp = pr.L, *Lb = pr.Lbar;
    double *Ab = pr.Abar;
    const long l1 = pr.ldl, l2 = pr.ldlb, l3 = pr.ldab;
    batched_trinv_lower(n, Lp, l1, X);
    __syncthreads();
    batched_prod(n, true, true, Lp, l1, false, true, Lb, l2, W, n);     // W = L^T Lbar
    __syncthreads();
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {      // Phi
      const int i = (int)(e % n), j = (int)(e / n);
      W[e] = i > j ? W[e] : (i == j ? 0.5 * W[e] : 0.0);
    }
    __syncthreads();
    batched_prod(n, false, false, W, n, false, true, X, n, Ab, l3);      // Abar = Phi L^-1
    __syncthreads();
    batched_prod(n, true, true, X, n, false, false, Ab, l3, W, n);       // W = L^-T Abar
    __syncthreads();
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {      // (S + S^T)/2
      const int i = (int)(e % n), j = (int)(e / n);
      Ab[i + (long)j * l3] = 0.5 * (W[i + (long)j * n] + W[j + (long)i * n]);
    }
    __syncthreads();
  }
}

// Bbar_p = A_p^-1 Xbar_p (A = L L^T, via L^-1), Abar_p -= (Bbar X^T + X Bbar^T)/2
// for every problem p (the unbatched atlb_dpotrs_adjoint_dev).
__global__ void __launch_bounds__(AT)
potrs_adjoint_batched_kernel(int count, const PotrsAdjProb *__restrict__ P, double *__restrict__ ws) {
  double *X = ws + (size_t)blockIdx.x * 2 * kAdjMaxN * kAdjMaxN;  // L^-1
  double *T = X + (size_t)kAdjMaxN * kAdjMaxN;                    // L^-1 Xbar
  for (int p = blockIdx.x; p < count; p += gridDim.x) {
    const PotrsAdjProb pr = P[p];
    const int n = pr.n, r = pr.nrhs;
    if (n <= 0 || n > kAdjMaxN || r <= 0 || r > kAdjMaxN) continue;
    const double *Lp = pr.L, *Xp = pr.X, *Xb = pr.Xbar;
    double *Bb = pr.Bbar, *Ab = pr.Abar;
    const long l1 = pr.ldl, lx = pr.ldx, lxb = pr.ldxb, lbb = pr.ldbb, lab = pr.ldab;
    batched_trinv_lower(n, Lp, l1, X);
    __syncthreads();
    for (long e = threadIdx.x; e < (long)n * r; e += blockDim.x) {  // T = L^-1 Xbar
      const int i = (int)(e % n), c = (int)(e / n);
      double s = 0.0;
      for (int k = 0; k <= i; k++) s = fma(X[i + (long)k * n], Xb[k + (long)c * lxb], s);
      T[i + (long)c * n] = s;
    }
    __syncthreads();
    for (long e = threadIdx.x; e < (long)n * r; e += blockDim.x) {  // Bbar = L^-T T
      const int i = (int)(e % n), c = (int)(e / n);
      double s = 0.0;
      for (int k = i; k < n; k++) s = fma(X[k + (long)i * n], T[k + (long)c * n], s);
      Bb[i + (long)c * lbb] = s;
    }
    __syncthreads();
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
      const int i = (int)(e % n), j = (int)(e / n);
      double s = 0.0;
      for (int c = 0; c < r; c++)
        s += Bb[i + (long)c * lbb] * Xp[j + (long)c * lx] + Xp[i + (long)c * lx] * Bb[j + (long)c * lbb];
      Ab[i + (long)j * lab] -= 0.5 * s;
    }
    __syncthreads();
  }
}

// the problem list on the device (pageable source: the copy has taken the
// host data when cudaMemcpyAsync returns, so the caller's arrays may change)
template <typename P>
const P *upload_probs(const std::vector<P> &v, int slot, cudaStream_t st) {
  P *d = (P *)scratch(slot, sizeof(P) * v.size());
  ATLB_CUDA_CHECK(cudaMemcpyAsync(d, v.data(), sizeof(P) * v.size(), cudaMemcpyHostToDevice, st));
  return d;
}

int batched_grid(int count) { return std::max(1, std::min(count, num_sms() * 2)); }

}  // namespace
}  // namespace atlb

using namespace atlb;

extern "C" {

int atlb_dpotrf_adjoint_dev(int N, const double *L, int ldl, const double *Lbar, int ldlb, double *Abar,
                            int ldab) {
  if (N < 0) return -1;
  if (ldl < std::max(1, N)) return -3;
  if (ldlb < std::max(1, N)) return -5;
  if (ldab < std::max(1, N)) return -7;
  if (N == 0) return 0;
  cudaStream_t st = stream();
  const long nn = (long)N * N;
  double *W = (double *)scratch(kSlotAdj0, sizeof(double) * (size_t)nn);
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, Lbar, ldlb, W, N, kPartLower);       // W = Lbar
  dtrmm_dev(kLeft, kLower, kTrans, kNonUnit, N, N, 1.0, L, ldl, W, N, st);        // W = L^T Lbar
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, W, N, W, N, kPartPhi);                // W = Phi(W)
  trsm_dev<double>(kRight, kLower, kNoTrans, kNonUnit, N, N, 1.0, L, ldl, W, N, st);  // W L^-1
  trsm_dev<double>(kLeft, kLower, kTrans, kNonUnit, N, N, 1.0, L, ldl, W, N, st);     // L^-T W
  symmetrize_avg_kernel<<<gfor(nn), 256, 0, st>>>(N, W, N, Abar, ldab);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

int atlb_dpotrs_adjoint_dev(int N, int NRHS, const double *L, int ldl, const double *X, int ldx,
                            const double *Xbar, int ldxb, double *Bbar, int ldbb, double *Abar,
                            int ldab) {
  if (N < 0) return -1;
  if (NRHS < 0) return -2;
  if (ldl < std::max(1, N)) return -4;
  if (ldx < std::max(1, N)) return -6;
  if (ldxb < std::max(1, N)) return -8;
  if (ldbb < std::max(1, N)) return -10;
  if (ldab < std::max(1, N)) return -12;
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  copy_kernel<<<gfor((long)N * NRHS), 256, 0, st>>>(N, NRHS, Xbar, ldxb, Bbar, ldbb);
  potrs_dev<double>(kLower, N, NRHS, L, ldl, Bbar, ldbb, st);                     // Bbar = A^-1 Xbar
  dgemm_dev(kNoTrans, kTrans, N, N, NRHS, -0.5, Bbar, ldbb, X, ldx, 1.0, Abar, ldab, st);
  dgemm_dev(kNoTrans, kTrans, N, N, NRHS, -0.5, X, ldx, Bbar, ldbb, 1.0, Abar, ldab, st);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

int atlb_dgetrs_adjoint_dev(int N, int NRHS, const double *LU, int ldlu, const int *ipiv,
                            const double *X, int ldx, const double *Xbar, int ldxb, double *Bbar,
                            int ldbb, double *Abar, int ldab) {
  if (N < 0) return -1;
  if (NRHS < 0) return -2;
  if (ldlu < std::max(1, N)) return -4;
  if (ldx < std::max(1, N)) return -7;
  if (ldxb < std::max(1, N)) return -9;
  if (ldbb < std::max(1, N)) return -11;
  if (ldab < std::max(1, N)) return -13;
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  copy_kernel<<<gfor((long)N * NRHS), 256, 0, st>>>(N, NRHS, Xbar, ldxb, Bbar, ldbb);
  getrs_dev<double>(kTrans, N, NRHS, LU, ldlu, ipiv, Bbar, ldbb, st);             // Bbar = A^-T Xbar
  dgemm_dev(kNoTrans, kTrans, N, N, NRHS, -1.0, Bbar, ldbb, X, ldx, 1.0, Abar, ldab, st);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

int atlb_dgetrf_adjoint_dev(int N, const double *LU, int ldlu, const int *ipiv, const double *Lbar,
                            int ldlb, const double *Ubar, int ldub, double *Abar, int ldab) {
  if (N < 0) return -1;
  if (ldlu < std::max(1, N)) return -3;
  if (ldlb < std::max(1, N)) return -6;
  if (ldub < std::max(1, N)) return -8;
  if (ldab < std::max(1, N)) return -10;
  if (N == 0) return 0;
  cudaStream_t st = stream();
  const long nn = (long)N * N;
  double *W1 = (double *)scratch(kSlotAdj0, sizeof(double) * (size_t)nn);
  double *W2 = (double *)scratch(kSlotAdj1, sizeof(double) * (size_t)nn);
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, Lbar, ldlb, W1, N, kPartStrictLower);  // W1 = stril(Lbar)
  dtrmm_dev(kLeft, kLower, kTrans, kUnit, N, N, 1.0, LU, ldlu, W1, N, st);         // W1 = L^T Lbar
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, W1, N, W1, N, kPartStrictLower);
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, Ubar, ldub, W2, N, kPartUpper);        // W2 = triu(Ubar)
  dtrmm_dev(kRight, kUpper, kTrans, kNonUnit, N, N, 1.0, LU, ldlu, W2, N, st);     // W2 = Ubar U^T
  part_kernel<<<gfor(nn), 256, 0, st>>>(N, W2, N, W2, N, kPartUpper);
  add_kernel<<<gfor(nn), 256, 0, st>>>(N, W1, N, W2, N, Abar, ldab);              // M
  trsm_dev<double>(kLeft, kLower, kTrans, kUnit, N, N, 1.0, LU, ldlu, Abar, ldab, st);     // L^-T M
  trsm_dev<double>(kRight, kUpper, kTrans, kNonUnit, N, N, 1.0, LU, ldlu, Abar, ldab, st); // ... U^-T
  laswp_dev<double>(N, Abar, ldab, 0, N, ipiv, -1, st);                             // P (...)
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

int atlb_dpotrf_adjoint_batched_dev(int count, const int *n, const double *const *L, const int *ldl,
                                    const double *const *Lbar, const int *ldlb, double *const *Abar,
                                    const int *ldab) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  std::vector<PotrfAdjProb> v(count);
  for (int i = 0; i < count; i++) {
    if (n[i] < 0 || n[i] > kAdjMaxN) return -2;
    if (ldl[i] < std::max(1, n[i])) return -4;
    if (ldlb[i] < std::max(1, n[i])) return -6;
    if (ldab[i] < std::max(1, n[i])) return -8;
    v[i] = {L[i], Lbar[i], Abar[i], n[i], ldl[i], ldlb[i], ldab[i]};
  }
  cudaStream_t st = stream();
  const int g = batched_grid(count);
  const PotrfAdjProb *dp = upload_probs(v, kSlotAdjProbs, st);
  double *ws = (double *)scratch(kSlotAdj2, sizeof(double) * (size_t)g * 2 * kAdjMaxN * kAdjMaxN);
  potrf_adjoint_batched_kernel<<<g, AT, 0, st>>>(count, dp, ws);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

int atlb_dpotrs_adjoint_batched_dev(int count, const int *n, const int *nrhs, const double *const *L,
                                    const int *ldl, const double *const *X, const int *ldx,
                                    const double *const *Xbar, const int *ldxb, double *const *Bbar,
                                    const int *ldbb, double *const *Abar, const int *ldab) {
  if (count < 0) return -1;
  if (count == 0) return 0;
  std::vector<PotrsAdjProb> v(count);
  for (int i = 0; i < count; i++) {
    if (n[i] < 0 || n[i] > kAdjMaxN) return -2;
    if (nrhs[i] < 0 || nrhs[i] > kAdjMaxN) return -3;
    if (ldl[i] < std::max(1, n[i])) return -5;
    if (ldx[i] < std::max(1, n[i])) return -7;
    if (ldxb[i] < std::max(1, n[i])) return -9;
    if (ldbb[i] < std::max(1, n[i])) return -11;
    if (ldab[i] < std::max(1, n[i])) return -13;
    v[i] = {L[i], X[i], Xbar[i], Bbar[i], Abar[i], n[i], nrhs[i], ldl[i], ldx[i], ldxb[i], ldbb[i], ldab[i]};
  }
  cudaStream_t st = stream();
  const int g = batched_grid(count);
  const PotrsAdjProb *dp = upload_probs(v, kSlotAdjProbs, st);
  double *ws = (double *)scratch(kSlotAdj2, sizeof(double) * (size_t)g * 2 * kAdjMaxN * kAdjMaxN);
  potrs_adjoint_batched_kernel<<<g, AT, 0, st>>>(count, dp, ws);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return 0;
}

}  // extern "C"
