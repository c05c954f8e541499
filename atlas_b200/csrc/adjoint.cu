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

}  // extern "C"
