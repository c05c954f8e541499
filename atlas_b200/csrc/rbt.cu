// Random butterfly transformation (RBT) for the mixed-precision solver.
// No counterpart in the reference.
//
// A x = b is replaced by (U^T A V) y = U^T b, x = V y, with U, V random
// recursive butterflies of depth 2 (Parker, 1995; Baboulin, Dongarra et al.):
// B = 1/sqrt(2) [[R0, R1], [R0, -R1]], R0/R1 diagonal with entries exp(r/10),
// r uniform in [-1/2, 1/2]; U = U1 U2 with U1 one butterfly of order n and U2
// two butterflies of order n/2 (same for V).  With high probability the
// transformed matrix can be factored without pivoting, which removes the
// column-by-column pivot search from the FP32 factorization; the FP64
// refinement against the original A recovers the accuracy, and if the
// factorization is unusable the solver falls back to FP64 partial pivoting.
//
// n is padded to a multiple of 4 with an identity block.  Each output element
// of U^T A V depends on one "quad" of 4 rows x 4 columns of A (rows i0 +
// {0, n/4, n/2, 3n/4}), so one thread transforms a whole 4x4 quad: every
// element of A is read once and every element of the result written once.
#include <algorithm>
#include <cmath>
#include "common.cuh"
#include "kernels.h"
#include "mixed.h"

namespace atlb {
namespace {

__device__ __forceinline__ double rbt_rand(uint64_t seed, uint64_t i) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + i + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;  // [-1/2, 1/2)
  return exp(u / 10.0);
}

// d[0..2n): per side, level-1 diagonals P0 (h), P1 (h), level-2 Q0a, Q1a,
// Q0b, Q1b (h/2 each); side 0 = U, side 1 = V
__global__ void rbt_init_kernel(int n, uint64_t seed, double *d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * n; i += gridDim.x * blockDim.x)
    d[i] = rbt_rand(seed, (uint64_t)i);
}

struct Quad {  // the four indices of a quad and their diagonal factors
  const double *P0, *P1, *Q0a, *Q1a, *Q0b, *Q1b;
};
__device__ __forceinline__ Quad quad_of(const double *d, int n) {
  const int h = n / 2, h2 = n / 4;
  Quad q;
  q.P0 = d; q.P1 = d + h; q.Q0a = d + n; q.Q1a = d + n + h2; q.Q0b = d + n + 2 * h2; q.Q1b = d + n + 3 * h2;
  return q;
}

// y = U^T a on the quad (a0 = a[i0], a1 = a[i0+h2], a2 = a[i0+h], a3 = a[i0+h+h2]);
// also the action of B applied from the right to a row vector.
__device__ __forceinline__ void bt_quad(const Quad &q, int i0, int h2, double (&a)[4]) {
  const double s = 0.70710678118654752440;
  // level 1: pairs (i, i+h) for i = i0 and i0 + h2
  double t0 = q.P0[i0] * (a[0] + a[2]) * s, t2 = q.P1[i0] * (a[0] - a[2]) * s;
  double t1 = q.P0[i0 + h2] * (a[1] + a[3]) * s, t3 = q.P1[i0 + h2] * (a[1] - a[3]) * s;
  // level 2: first half pairs (t0, t1), second half pairs (t2, t3)
  a[0] = q.Q0a[i0] * (t0 + t1) * s;
  a[1] = q.Q1a[i0] * (t0 - t1) * s;
  a[2] = q.Q0b[i0] * (t2 + t3) * s;
  a[3] = q.Q1b[i0] * (t2 - t3) * s;
}

// x = V y on the quad (inverse order of the levels, B itself)
__device__ __forceinline__ void b_quad(const Quad &q, int i0, int h2, double (&y)[4]) {
  const double s = 0.70710678118654752440;
  // level 2: x_half = B_half y_half
  double t0 = (q.Q0a[i0] * y[0] + q.Q1a[i0] * y[1]) * s, t1 = (q.Q0a[i0] * y[0] - q.Q1a[i0] * y[1]) * s;
  double t2 = (q.Q0b[i0] * y[2] + q.Q1b[i0] * y[3]) * s, t3 = (q.Q0b[i0] * y[2] - q.Q1b[i0] * y[3]) * s;
  // level 1: pairs (i, i+h): (t0, t2) at i0 and (t1, t3) at i0 + h2
  y[0] = (q.P0[i0] * t0 + q.P1[i0] * t2) * s;
  y[2] = (q.P0[i0] * t0 - q.P1[i0] * t2) * s;
  y[1] = (q.P0[i0 + h2] * t1 + q.P1[i0 + h2] * t3) * s;
  y[3] = (q.P0[i0 + h2] * t1 - q.P1[i0 + h2] * t3) * s;
}

// S (n4 x n4, FP32, ld n4) = U^T A_pad V, A (n x n FP64, lda)
__global__ void rbt_matrix_kernel(int n, int n4, const double *__restrict__ A, long lda,
                                  const double *__restrict__ du, const double *__restrict__ dv,
                                  float *__restrict__ S) {
  const int h2 = n4 / 4;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x, j0 = blockIdx.y;
  if (i0 >= h2 || j0 >= h2) return;
  const Quad qu = quad_of(du, n4), qv = quad_of(dv, n4);
  const int ri[4] = {i0, i0 + h2, i0 + 2 * h2, i0 + 3 * h2};
  const int cj[4] = {j0, j0 + h2, j0 + 2 * h2, j0 + 3 * h2};
  double m[4][4];  // m[r][c]
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int i = ri[r], j = cj[c];
      m[r][c] = (i < n && j < n) ? A[i + (long)j * lda] : (i == j ? 1.0 : 0.0);
    }
  // rows: U^T on each column of the quad
#pragma unroll
  for (int c = 0; c < 4; c++) {
    double a[4] = {m[0][c], m[1][c], m[2][c], m[3][c]};
    bt_quad(qu, i0, h2, a);
#pragma unroll
    for (int r = 0; r < 4; r++) m[r][c] = a[r];
  }
  // columns: times V on each row of the quad (same formula as U^T on a vector)
#pragma unroll
  for (int r = 0; r < 4; r++) {
    double a[4] = {m[r][0], m[r][1], m[r][2], m[r][3]};
    bt_quad(qv, j0, h2, a);
#pragma unroll
    for (int c = 0; c < 4; c++) S[ri[r] + (long)cj[c] * n4] = (float)a[c];
  }
}

// C (n4 x nrhs, FP32) = U^T r_pad, r (n x nrhs FP64)
__global__ void rbt_left_vec_kernel(int n, int n4, int nrhs, const double *__restrict__ R, long ldr,
                                    const double *__restrict__ du, float *__restrict__ C) {
  const int h2 = n4 / 4, i0 = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y;
  if (i0 >= h2 || q >= nrhs) return;
  const Quad qu = quad_of(du, n4);
  double a[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int i = i0 + r * h2;
    a[r] = i < n ? R[i + (long)q * ldr] : 0.0;
  }
  bt_quad(qu, i0, h2, a);
#pragma unroll
  for (int r = 0; r < 4; r++) C[i0 + r * h2 + (long)q * n4] = (float)a[r];
}

// X (n x nrhs FP64) += (V y)[0:n], y (n4 x nrhs FP32)
__global__ void rbt_right_add_kernel(int n, int n4, int nrhs, const float *__restrict__ Y,
                                     const double *__restrict__ dv, double *__restrict__ X, long ldx) {
  const int h2 = n4 / 4, i0 = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y;
  if (i0 >= h2 || q >= nrhs) return;
  const Quad qv = quad_of(dv, n4);
  double y[4];
#pragma unroll
  for (int r = 0; r < 4; r++) y[r] = (double)Y[i0 + r * h2 + (long)q * n4];
  b_quad(qv, i0, h2, y);
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int i = i0 + r * h2;
    if (i < n) X[i + (long)q * ldx] += y[r];
  }
}

}  // namespace

int rbt_order(int n) { return (n + 3) / 4 * 4; }

// Random diagonals of U (d) and V (d + 2*n4), deterministic for a given n4.
void rbt_init_dev(int n4, double *d, cudaStream_t st) {
  rbt_init_kernel<<<std::min(cdiv(4L * n4, 256), 1024), 256, 0, st>>>(n4, 0x5EEDB0DDull + (uint64_t)n4, d);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void rbt_matrix_dev(int n, const double *A, long lda, const double *d, float *S, cudaStream_t st) {
  const int n4 = rbt_order(n), h2 = n4 / 4;
  rbt_matrix_kernel<<<dim3(cdiv(h2, 128), h2), 128, 0, st>>>(n, n4, A, lda, d, d + 2 * n4, S);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void rbt_left_vec_dev(int n, int nrhs, const double *R, long ldr, const double *d, float *C,
                      cudaStream_t st) {
  const int n4 = rbt_order(n), h2 = n4 / 4;
  rbt_left_vec_kernel<<<dim3(cdiv(h2, 256), nrhs), 256, 0, st>>>(n, n4, nrhs, R, ldr, d, C);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void rbt_right_add_dev(int n, int nrhs, const float *Y, const double *d, double *X, long ldx,
                       cudaStream_t st) {
  const int n4 = rbt_order(n), h2 = n4 / 4;
  rbt_right_add_kernel<<<dim3(cdiv(h2, 256), nrhs), 256, 0, st>>>(n, n4, nrhs, Y, d + 2 * n4, X, ldx);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

}  // namespace atlb
