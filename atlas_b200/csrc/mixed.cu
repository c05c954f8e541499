// Mixed-precision solvers: factor in FP32 on the GPU (trailing updates on the
// tensor cores in TF32 or BF16 with FP32 accumulation, or exact FP32 FMA),
// recover FP64 accuracy by iterative refinement.  FP64 is used only for the
// residual r = b - A x, the solution update and the norms that decide
// convergence.  No counterpart in the reference (ATLAS has no mixed-precision
// solver); the interface and the fallback rule follow LAPACK's dsgesv /
// dsposv: A and B are left unchanged when refinement succeeds; if it does
// not converge (or the FP32 factorization breaks down) the FP64 solver is
// used and `iter` is returned negative.
//
// Stopping rule: every right-hand side reaches a normwise backward error
// ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= N * 2^-53.
#include <algorithm>
#include <cmath>
#include <vector>
#include "common.cuh"
#include "kernels.h"
#include "mixed.h"
#include "staging.h"
#include "../../include/atlas_b200.h"

namespace atlb {
namespace {

constexpr int ITERMAX = 30;

__global__ void d2s_kernel(int M, int N, const double *__restrict__ A, long lda, float *__restrict__ S,
                           long lds) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    S[i + (long)j * lds] = (float)A[i + (long)j * lda];
  }
}

__global__ void add_s2d_kernel(int M, int N, const float *__restrict__ S, long lds, double *__restrict__ X,
                               long ldx) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    X[i + (long)j * ldx] += (double)S[i + (long)j * lds];
  }
}

// S(i, j) = (float) R(perm[i], j): the row interchanges fused into the conversion
__global__ void gather_d2s_kernel(int M, int N, const double *__restrict__ R, long ldr,
                                  const int *__restrict__ perm, float *__restrict__ S, long lds) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    S[i + (long)j * lds] = (float)R[perm[i] + (long)j * ldr];
  }
}

__global__ void s2d_kernel(int M, int N, const float *__restrict__ S, long lds, double *__restrict__ X,
                           long ldx) {
  long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % M), j = (int)(idx / M);
    X[i + (long)j * ldx] = (double)S[i + (long)j * lds];
  }
}

// partial row sums of |A| over column chunks: part[chunk * N + i]
constexpr int GV_ROWS = 256, GV_COLS = 256;
__global__ void __launch_bounds__(GV_ROWS)
abs_rowsum_partial_kernel(int N, const double *__restrict__ A, long lda, double *__restrict__ part) {
  const int i = blockIdx.x * GV_ROWS + threadIdx.x, c0 = blockIdx.y * GV_COLS;
  if (i >= N) return;
  double s = 0.0;
  const int c1 = min(N, c0 + GV_COLS);
  for (int c = c0; c < c1; c++) s += fabs(A[i + (long)c * lda]);
  part[(long)blockIdx.y * N + i] = s;
}

// S = (float) A and abs_rowsum_partial_kernel's partials in one pass over A
// (the mixed solvers need both before factoring): per 256-column chunk, thread
// i converts its row's elements and sums their magnitudes in column order,
// the order of abs_rowsum_partial_kernel, eight loads in flight.
__global__ void __launch_bounds__(GV_ROWS)
d2s_rowsum_kernel(int N, int ncols, const double *__restrict__ A, long lda, float *__restrict__ S, long lds,
                  double *__restrict__ part) {
  const int i = blockIdx.x * GV_ROWS + threadIdx.x, c0 = blockIdx.y * GV_COLS;
  if (i >= N) return;
  const int c1 = min(ncols, c0 + GV_COLS);
  const double *a = A + i + (long)c0 * lda;
  float *o = S + i + (long)c0 * lds;
  double s = 0.0;
  int c = c0;
  for (; c + 8 <= c1; c += 8, a += 8 * lda, o += 8 * lds) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = a[(long)q * lda];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      o[(long)q * lds] = (float)v[q];
      s += fabs(v[q]);
    }
  }
  for (; c < c1; c++, a += lda, o += lds) {
    const double v = *a;
    *o = (float)v;
    s += fabs(v);
  }
  part[(long)blockIdx.y * N + i] = s;
}

// residual partials: part[(chunk * nrhs + r) * N + i] = sum_{c in chunk} A(i,c) X(c,r)
template <int NR>
__global__ void __launch_bounds__(GV_ROWS)
gemv_partial_kernel(int N, int nrhs, const double *__restrict__ A, long lda,
                    const double *__restrict__ X, long ldx, double *__restrict__ part) {
  __shared__ double xs[GV_COLS][NR];
  const int c0 = blockIdx.y * GV_COLS, i = blockIdx.x * GV_ROWS + threadIdx.x;
  const int c1 = min(N, c0 + GV_COLS);
  for (int t = threadIdx.x; t < GV_COLS * NR; t += GV_ROWS) {
    int c = t / NR, r = t % NR;
    xs[c][r] = (c0 + c < N && r < nrhs) ? X[(c0 + c) + (long)r * ldx] : 0.0;
  }
  __syncthreads();
  if (i >= N) return;
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) acc[r] = 0.0;
  const double *a = A + i + (long)c0 * lda;
  int c = c0;
  for (; c + 4 <= c1; c += 4) {
    double a0 = a[0], a1 = a[lda], a2 = a[2 * lda], a3 = a[3 * lda];
    const int k = c - c0;
#pragma unroll
    for (int r = 0; r < NR; r++)
      acc[r] = fma(a3, xs[k + 3][r], fma(a2, xs[k + 2][r], fma(a1, xs[k + 1][r], fma(a0, xs[k][r], acc[r]))));
    a += 4 * lda;
  }
  for (; c < c1; c++) {
    const double av = a[0];
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r] = fma(av, xs[c - c0][r], acc[r]);
    a += lda;
  }
#pragma unroll
  for (int r = 0; r < NR; r++)
    if (r < nrhs) part[((long)blockIdx.y * nrhs + r) * N + i] = acc[r];
}

// R = B - sum of partials (fixed order: deterministic); also per-RHS maxima of
// |R| and |X| and |B| into red[3*r + {0,1,2}] via atomicMax on the bit patterns
__global__ void resid_finish_kernel(int N, int nrhs, int nchunks, const double *__restrict__ part,
                                    const double *__restrict__ B, long ldb,
                                    const double *__restrict__ X, long ldx, double *__restrict__ R,
                                    long ldr, unsigned long long *__restrict__ red) {
  const int r = blockIdx.y;
  double mr = 0.0, mx = 0.0, mb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += part[((long)ch * nrhs + r) * N + i];
    const double b = B[i + (long)r * ldb];
    const double v = b - s;
    const double xv = X[i + (long)r * ldx];
    R[i + (long)r * ldr] = v;
    // NaN must not vanish in the maximum (fmax drops it): count it as infinite
    mr = fmax(mr, v == v ? fabs(v) : INFINITY);
    mx = fmax(mx, xv == xv ? fabs(xv) : INFINITY);
    mb = fmax(mb, fabs(b));
  }
  for (int o = 16; o; o >>= 1) {
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
  }
  if ((threadIdx.x & 31) == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax(&red[3 * r + 0], (unsigned long long)__double_as_longlong(mr));
    atomicMax(&red[3 * r + 1], (unsigned long long)__double_as_longlong(mx));
    atomicMax(&red[3 * r + 2], (unsigned long long)__double_as_longlong(mb));
  }
}

__global__ void rowsum_finish_kernel(int N, int nchunks, const double *__restrict__ part,
                                     unsigned long long *__restrict__ out) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += part[(long)ch * N + i];
    m = fmax(m, s);
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void symmetrize_kernel(int uplo, int N, const double *__restrict__ A, long lda,
                                  double *__restrict__ F, long ldf) {
  long total = (long)N * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    int i = (int)(idx % N), j = (int)(idx / N);
    bool stored = (uplo == kLower) ? (i >= j) : (i <= j);
    F[i + (long)j * ldf] = stored ? A[i + (long)j * lda] : A[j + (long)i * lda];
  }
}

// ---- GMRES-based refinement kernels (FP64 vectors of length N, nrhs columns
// iterated in lockstep; the Krylov basis V holds vector i of column c at
// V + (i * nrhs + c) * N).

// Y = sum of the GEMV partials (fixed order)
__global__ void gemv_sum_kernel(int N, int nrhs, int nchunks, const double *__restrict__ part,
                                double *__restrict__ Y, long ldy) {
  const int r = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += part[((long)ch * nrhs + r) * N + i];
    Y[i + (long)r * ldy] = s;
  }
}

// h[i * nrhs + c] = <V_i[:, c], W[:, c]> for i < gridDim.x, one CTA per (i, c)
__global__ void __launch_bounds__(256) multidot_kernel(int N, int nrhs, const double *__restrict__ V,
                                                       const double *__restrict__ W, double *__restrict__ h) {
  __shared__ double red[8];
  const int i = blockIdx.x, c = blockIdx.y;
  const double *v = V + ((long)i * nrhs + c) * N, *w = W + (long)c * N;
  double s = 0.0;
  for (int r = threadIdx.x; r < N; r += 256) s = fma(v[r], w[r], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < 8; q++) t += red[q];
    h[(long)i * nrhs + c] = t;
  }
}

// X[:, c] += sgn * sum_{i < k} V_i[:, c] y[i * nrhs + c]
__global__ void vcombine_kernel(int N, int nrhs, int k, const double *__restrict__ V, const double *__restrict__ y,
                                double sgn, double *__restrict__ X, long ldx) {
  const int c = blockIdx.y;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < k; i++) s = fma(V[((long)i * nrhs + c) * N + r], y[(long)i * nrhs + c], s);
    X[r + (long)c * ldx] += sgn * s;
  }
}

// Vout[:, c] = W[:, c] / sqrt(nrm2[c]) (zero for a zero norm)
__global__ void vscale_kernel(int N, int nrhs, const double *__restrict__ W, const double *__restrict__ nrm2,
                              double *__restrict__ Vout) {
  const int c = blockIdx.y;
  const double q = nrm2[c] > 0.0 ? 1.0 / sqrt(nrm2[c]) : 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x)
    Vout[(long)c * N + r] = W[(long)c * N + r] * q;
}

bool debug_ir() {
  static int v = -1;
  if (v < 0) { const char *e = getenv("ATLAS_B200_DEBUG_IR"); v = (e && *e && *e != '0') ? 1 : 0; }
  return v == 1;
}

inline int grid_for(long total) { return (int)std::min<long>((total + 255) / 256, 148L * 8); }

}  // namespace

void symmetrize_dev(int uplo, int N, const double *A, long lda, double *F, long ldf, cudaStream_t st) {
  symmetrize_kernel<<<grid_for((long)N * N), 256, 0, st>>>(uplo, N, A, lda, F, ldf);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// The factorization's GEMMs: the tensor-core paths pay an operand
// conversion pass per call, which only large updates (the block trailing
// updates, K >= 256) amortize; the small updates inside a block column run
// as plain FP32 FMA GEMMs (more accurate than the tensor-core formats, so the
// factorization is at least as accurate as with the tensor cores alone).
template <void (*TC)(int, int, int, int, int, float, const float *, long, const float *, long, float,
                     float *, long, cudaStream_t, int)>
void sgemm_by_size(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                   const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st, int tri) {
  if (K < 128 || (long)M * N * K < (1L << tune(kTuneTcMinWorkLog2)))
    sgemm_dev(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
  else
    TC(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, st, tri);
}

SgemmFn factor_gemm(int prec) {
  if (prec == kPrecTF32) return sgemm_by_size<sgemm_tf32_dev>;
  if (prec == kPrecBF16) return sgemm_by_size<sgemm_bf16_dev>;
  if (prec == kPrecTF32x3) return sgemm_by_size<sgemm_tf32x3_dev>;
  return sgemm_dev;
}

// ||A||_inf (FP64) into *out (device, as bits), using part (N * ceil(N/256) doubles)
void dnorm_inf_dev(int N, const double *A, long lda, double *part, unsigned long long *out,
                   cudaStream_t st) {
  const int nch = cdiv(N, GV_COLS);
  ATLB_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  abs_rowsum_partial_kernel<<<dim3(cdiv(N, GV_ROWS), nch), GV_ROWS, 0, st>>>(N, A, lda, part);
  rowsum_finish_kernel<<<std::min(cdiv(N, 256), 148), 256, 0, st>>>(N, nch, part, out);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// R = B - A X; red[3r..3r+2] = max|R_r|, max|X_r|, max|B_r| (right-hand
// sides are processed 8 at a time; part holds ceil(N/256) * 8 * N doubles)
void dresid_dev(int N, int nrhs, const double *A, long lda, const double *X, long ldx,
                const double *B, long ldb, double *R, long ldr, double *part,
                unsigned long long *red, cudaStream_t st) {
  const int nch = cdiv(N, GV_COLS);
  ATLB_CUDA_CHECK(cudaMemsetAsync(red, 0, sizeof(unsigned long long) * 3 * nrhs, st));
  dim3 grid(cdiv(N, GV_ROWS), nch);
  for (int r0 = 0; r0 < nrhs; r0 += 8) {
    const int nr = std::min(8, nrhs - r0);
    const double *Xr = X + (long)r0 * ldx;
    if (nr <= 1) gemv_partial_kernel<1><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, ldx, part);
    else if (nr <= 4) gemv_partial_kernel<4><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, ldx, part);
    else gemv_partial_kernel<8><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, ldx, part);
    resid_finish_kernel<<<dim3(std::min(cdiv(N, 256), 64), nr), 256, 0, st>>>(
        N, nr, nch, part, B + (long)r0 * ldb, ldb, Xr, ldx, R + (long)r0 * ldr, ldr, red + 3 * r0);
  }
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// S = (float) A (N x N) and ||A||_inf into *out (as dnorm_inf_dev), one pass over A
void d2s_norm_dev(int N, const double *A, long lda, float *S, long lds, double *part, unsigned long long *out,
                  cudaStream_t st) {
  const int nch = cdiv(N, GV_COLS);
  ATLB_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  d2s_rowsum_kernel<<<dim3(cdiv(N, GV_ROWS), nch), GV_ROWS, 0, st>>>(N, N, A, lda, S, lds, part);
  rowsum_finish_kernel<<<std::min(cdiv(N, 256), 148), 256, 0, st>>>(N, nch, part, out);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// d2s_rowsum_kernel with the rows gathered: row i of S takes row perm[i] of
// A, whose row-sum partial goes to part[.. + perm[i]] (the partial belongs to
// the source row, so the norm does not depend on the order).
__global__ void __launch_bounds__(GV_ROWS)
d2s_rowsum_perm_kernel(int N, int ncols, const double *__restrict__ A, long lda, const int *__restrict__ perm,
                       float *__restrict__ S, long lds, double *__restrict__ part) {
  const int i = blockIdx.x * GV_ROWS + threadIdx.x, c0 = blockIdx.y * GV_COLS;
  if (i >= N) return;
  const int c1 = min(ncols, c0 + GV_COLS), src = perm[i];
  const double *a = A + src + (long)c0 * lda;
  float *o = S + i + (long)c0 * lds;
  double s = 0.0;
  int c = c0;
  for (; c + 8 <= c1; c += 8, a += 8 * lda, o += 8 * lds) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = a[(long)q * lda];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      o[(long)q * lds] = (float)v[q];
      s += fabs(v[q]);
    }
  }
  for (; c < c1; c++, a += lda, o += lds) {
    const double v = *a;
    *o = (float)v;
    s += fabs(v);
  }
  part[(long)blockIdx.y * N + src] = s;
}

// out[i] = ipiv[i] for i < h, i (no interchange) for h <= i < n
__global__ void head_ipiv_kernel(int n, int h, const int *__restrict__ ipiv, int *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i < h ? ipiv[i] : i;
}

// Y (M x ncols) = rows perm[0..M) of X
__global__ void gather_rows_kernel(int M, int ncols, const float *__restrict__ X, long ldx,
                                   const int *__restrict__ perm, float *__restrict__ Y, long ldy) {
  const long total = (long)M * ncols;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % M), j = (int)(idx / M);
    Y[i + (long)j * ldy] = X[perm[i] + (long)j * ldx];
  }
}

// Pivot numbers of the trailing factorization made absolute (ipiv[h..n) +=
// h), and its info (dinfo2: 0 or its first zero pivot, counted from row h)
// folded into *dinfo when the leading part had none.
__global__ void split_fixup_kernel(int n, int h, int *ipiv, int *dinfo, const int *dinfo2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (h + i < n) ipiv[h + i] += h;
  if (i == 0 && *dinfo == 0 && *dinfo2 > 0) *dinfo = h + *dinfo2;
}

// B = L^-1 B for L unit lower triangular (n x n) and B n x m, n a multiple
// of 256 (or at most 256): halves at multiples of 256 down to 256-row
// leaves, each solved in one trsm_llu_small_dev launch, the halves coupled by
// one GEMM per level (K >= 256, so every product runs at the tensor cores'
// long-K rate; trsm_dev's 64-row leaves suit narrow right-hand sides).
void llu_solve(int n, int m, const float *L, long ldl, float *B, long ldb, SgemmFn gemm, cudaStream_t st) {
  if (n <= 256) {
    trsm_llu_small_dev<float>(n, m, L, ldl, B, ldb, st);
    return;
  }
  const int n1 = (n / 2 + 255) / 256 * 256;
  llu_solve(n1, m, L, ldl, B, ldb, gemm, st);
  (gemm ? gemm : sgemm_dev)(kNoTrans, kNoTrans, n - n1, m, n1, -1.f, L + n1, ldl, B, ldb, 1.f, B + n1, ldb, st, 0);
  llu_solve(n - n1, m, L + n1 + (long)n1 * ldl, ldl, B + n1, ldb, gemm, st);
}

// The FP32 factorization of a host matrix overlapped with its copy, as the
// outer levels of src/lapack/ATL_getrfC.c's recursion taken left to right
// over column segments [0, N/16), [N/16, N/8), [N/8, N/4), [N/4, N/2),
// [N/2, N) (block columns of GV_COLS).
// The copy stream brings the block columns over back to back.  The first
// segment is converted as its columns land (S and the row-sum partials) and
// factored (getrf_dev on its N-row panel) while the rest is still being
// copied.  Each later segment, once its columns have landed, is converted
// with the row interchanges of everything to its left applied (one gather
// through their net permutation), brought up to date with the factored
// columns in two large operations (the unit-lower solve of its top rows, the
// product with the L below), and its panel factored; its interchanges reach
// the L to its left by one gather of those rows.  ||A||_inf is summed from
// the partials at the end, as in d2s_norm_dev.  The copies start after the
// work already on st (a previous call may still read dA).
void streamed_factor_dev(int N, const double *hA, long hlda, double *dA, long dlda, float *S, long lds,
                         int *ipiv, int *dinfo, double *part, unsigned long long *nrm, SgemmFn gemm,
                         cudaStream_t st) {
  const int nblk = cdiv(N, GV_COLS);
  std::vector<int> segs = {0};
  for (int d : {16, 8, 4, 2})
    if (nblk / d * GV_COLS > segs.back()) segs.push_back(nblk / d * GV_COLS);
  segs.push_back(N);
  int *pw = (int *)scratch(kSlotStreamPerm, sizeof(int) * 2 * (size_t)N);
  int *head = pw, *perm = pw + N;
  float *tmp = (float *)scratch(kSlotStreamTmp, sizeof(float) * (size_t)(N / 2 + GV_COLS) * (N / 2 + GV_COLS));
  cudaStream_t cs = copy_stream();
  ATLB_CUDA_CHECK(cudaMemsetAsync(nrm, 0, sizeof(unsigned long long), st));
  ATLB_CUDA_CHECK(cudaEventRecord(chunk_event(0), st));
  ATLB_CUDA_CHECK(cudaStreamWaitEvent(cs, chunk_event(0), 0));
  for (int c = 0; c < nblk; c++) {
    const int c0 = c * GV_COLS, w = std::min(GV_COLS, N - c0);
    ATLB_CUDA_CHECK(cudaMemcpy2DAsync(dA + (long)c0 * dlda, dlda * sizeof(double), hA + (long)c0 * hlda,
                                      hlda * sizeof(double), (size_t)N * sizeof(double), w,
                                      cudaMemcpyHostToDevice, cs));
    ATLB_CUDA_CHECK(cudaEventRecord(chunk_event(1 + c), cs));
  }
  for (size_t si = 0; si + 1 < segs.size(); si++) {
    const int a = segs[si], b = segs[si + 1], w = b - a;
    if (w <= 0) continue;
    float *Sa = S + (long)a * lds;
    if (a == 0) {  // converted chunk by chunk as the columns land
      for (int c = 0; c < cdiv(b, GV_COLS); c++) {
        const int c0 = c * GV_COLS;
        ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, chunk_event(1 + c), 0));
        d2s_rowsum_kernel<<<dim3(cdiv(N, GV_ROWS), 1), GV_ROWS, 0, st>>>(
            N, std::min(GV_COLS, b - c0), dA + (long)c0 * dlda, dlda, S + (long)c0 * lds, lds, part + (long)c * N);
      }
      ATLB_CUDA_CHECK(cudaGetLastError());
      getrf_dev<float>(N, w, S, lds, ipiv, dinfo, st, gemm);
      continue;
    }
    // converted through the net permutation of ipiv[0..a), then updated
    head_ipiv_kernel<<<cdiv(N, 256), 256, 0, st>>>(N, a, ipiv, head);
    ipiv_to_perm_dev(N, head, perm, st);
    ATLB_CUDA_CHECK(cudaStreamWaitEvent(st, chunk_event(cdiv(b, GV_COLS)), 0));  // copies land in order
    d2s_rowsum_perm_kernel<<<dim3(cdiv(N, GV_ROWS), cdiv(w, GV_COLS)), GV_ROWS, 0, st>>>(
        N, w, dA + (long)a * dlda, dlda, perm, Sa, lds, part + (long)(a / GV_COLS) * N);
    ATLB_CUDA_CHECK(cudaGetLastError());
    llu_solve(a, w, S, lds, Sa, lds, gemm, st);
    (gemm ? gemm : sgemm_dev)(kNoTrans, kNoTrans, N - a, w, a, -1.f, S + a, lds, Sa, lds, 1.f, Sa + a, lds, st, 0);
    // its panel, then its interchanges on the L to its left (one gather)
    getrf_dev<float>(N - a, w, Sa + a, lds, ipiv + a, dinfo + 1, st, gemm);
    head_ipiv_kernel<<<cdiv(N - a, 256), 256, 0, st>>>(N - a, w, ipiv + a, head);  // its w pivots only
    ipiv_to_perm_dev(N - a, head, perm, st);
    gather_rows_kernel<<<grid_for((long)(N - a) * a), 256, 0, st>>>(N - a, a, S + a, lds, perm, tmp, N - a);
    ATLB_CUDA_CHECK(cudaMemcpy2DAsync(S + a, lds * sizeof(float), tmp, (N - a) * sizeof(float),
                                      (N - a) * sizeof(float), a, cudaMemcpyDeviceToDevice, st));
    split_fixup_kernel<<<cdiv(w, 256), 256, 0, st>>>(b, a, ipiv, dinfo, dinfo + 1);
  }
  rowsum_finish_kernel<<<std::min(cdiv(N, 256), 148), 256, 0, st>>>(N, nblk, part, nrm);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// The referenced triangle of S (uplo) copied, transposed, into the other
// one (the diagonal stays): after a Cholesky factorization S then holds L and
// L^T (or U^T and U), so both triangular solves read their factor with
// coalesced column accesses.  32 x 32 tiles through shared memory; a CTA
// takes the tile pair (bi, bj), bi > bj, of the lower grid.
__global__ void mirror_tri_kernel(int uplo, int N, float *__restrict__ S, long lds) {
  __shared__ float t[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  // source tile: rows of block bi, columns of block bj (lower) or its transpose position (upper)
  const int sr0 = uplo == kLower ? bi * 32 : bj * 32, sc0 = uplo == kLower ? bj * 32 : bi * 32;
  for (int q = ty; q < 32; q += 8) {
    const int r = sr0 + tx, c = sc0 + q;
    t[q][tx] = (r < N && c < N) ? S[r + (long)c * lds] : 0.f;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int r = sc0 + tx, c = sr0 + q;  // destination: the transposed position
    const bool strict = uplo == kLower ? r < c : r > c;
    if (r < N && c < N && strict) S[r + (long)c * lds] = t[tx][q];
  }
}

void d2s_dev(int M, int N, const double *A, long lda, float *S, long lds, cudaStream_t st) {
  d2s_kernel<<<grid_for((long)M * N), 256, 0, st>>>(M, N, A, lda, S, lds);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void gather_d2s_dev(int M, int N, const double *R, long ldr, const int *perm, float *S, long lds,
                    cudaStream_t st) {
  gather_d2s_kernel<<<grid_for((long)M * N), 256, 0, st>>>(M, N, R, ldr, perm, S, lds);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void s2d_dev(int M, int N, const float *S, long lds, double *X, long ldx, cudaStream_t st) {
  s2d_kernel<<<grid_for((long)M * N), 256, 0, st>>>(M, N, S, lds, X, ldx);
  ATLB_CUDA_CHECK(cudaGetLastError());
}
void add_s2d_dev(int M, int N, const float *S, long lds, double *X, long ldx, cudaStream_t st) {
  add_s2d_kernel<<<grid_for((long)M * N), 256, 0, st>>>(M, N, S, lds, X, ldx);
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// Y (N x nrhs, ld N) = A X (X: N x nrhs, ld N); part as for dresid_dev
void dgemv_dev(int N, int nrhs, const double *A, long lda, const double *X, double *Y, double *part,
               cudaStream_t st) {
  const int nch = cdiv(N, GV_COLS);
  dim3 grid(cdiv(N, GV_ROWS), nch);
  for (int r0 = 0; r0 < nrhs; r0 += 8) {
    const int nr = std::min(8, nrhs - r0);
    const double *Xr = X + (long)r0 * N;
    if (nr <= 1) gemv_partial_kernel<1><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, N, part);
    else if (nr <= 4) gemv_partial_kernel<4><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, N, part);
    else gemv_partial_kernel<8><<<grid, GV_ROWS, 0, st>>>(N, nr, A, lda, Xr, N, part);
    gemv_sum_kernel<<<dim3(std::min(cdiv(N, 256), 64), nr), 256, 0, st>>>(N, nr, nch, part, Y + (long)r0 * N, N);
  }
  ATLB_CUDA_CHECK(cudaGetLastError());
}

// One GMRES-IR correction (Carson & Higham, "Accelerating the solution of
// linear systems by iterative refinement in three precisions", SIAM J. Sci.
// Comput. 40(2), 2018; on GPUs with a tensor-core LU, Haidar, Tomov,
// Dongarra & Higham, SC18): X += d, d from GMRES on the left-preconditioned
// system M^-1 A d = M^-1 R, M = the low-precision factors (`correct` applies
// M^-1 to a zeroed vector), FP64 Arnoldi with classical Gram-Schmidt
// repeated once (CGS2), Givens rotations and the small least-squares solve on
// the host.  Stops when every column's preconditioned residual estimate has
// dropped by KRYLOV_TAU or after KRYLOV_M steps; returns the steps taken.
// When u_low * kappa(A) is near or above 1, plain refinement (one M^-1 solve
// per step) stagnates or diverges while this correction still converges.
constexpr int KRYLOV_M = 30;
constexpr int KRYLOV_MAX_RHS = 8;
constexpr double KRYLOV_TAU = 1e-4;

template <class Correct>
int gmres_correct(int N, int nrhs, const double *A, long lda, const double *R, long ldr, double *X, long ldx,
                  Correct correct, double *part, cudaStream_t st) {
  const int m = KRYLOV_M;
  const size_t nv = (size_t)N * nrhs;
  double *V = (double *)scratch(kSlotKrylov, sizeof(double) * (nv * (m + 3) + (size_t)(3 * (m + 1) + m + 1) * nrhs));
  double *Z = V + nv * (m + 1), *Wv = Z + nv;
  double *h1 = Wv + nv, *h2 = h1 + (size_t)(m + 1) * nrhs, *nrm = h2 + (size_t)(m + 1) * nrhs;
  double *y = nrm + nrhs;
  double *hh = (double *)pinned(kSlotKrylovH, sizeof(double) * (size_t)(3 * (m + 1) + m + 1) * nrhs);
  double *hh1 = hh, *hh2 = hh1 + (size_t)(m + 1) * nrhs, *hnrm = hh2 + (size_t)(m + 1) * nrhs,
         *hy = hnrm + nrhs;
  const dim3 vgrid(std::min(cdiv(N, 256), 148), nrhs);
  // v0 = M^-1 R / beta
  ATLB_CUDA_CHECK(cudaMemsetAsync(V, 0, sizeof(double) * nv, st));
  correct(R, ldr, V, N);
  multidot_kernel<<<dim3(1, nrhs), 256, 0, st>>>(N, nrhs, V, V, nrm);
  vscale_kernel<<<vgrid, 256, 0, st>>>(N, nrhs, V, nrm, V);
  ATLB_CUDA_CHECK(cudaGetLastError());
  ATLB_CUDA_CHECK(cudaMemcpyAsync(hnrm, nrm, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  std::vector<double> H((size_t)nrhs * (m + 1) * m, 0.0), g((size_t)nrhs * (m + 1), 0.0), cs((size_t)nrhs * m),
      sn((size_t)nrhs * m), beta(nrhs);
  auto Hc = [&](int c, int i, int j) -> double & { return H[((size_t)c * (m + 1) + i) * m + j]; };
  for (int c = 0; c < nrhs; c++) {
    beta[c] = std::sqrt(std::max(hnrm[c], 0.0));
    g[(size_t)c * (m + 1)] = beta[c];
  }
  int j = 0;
  while (j < m) {
    const double *Vj = V + (size_t)j * nv;
    double *Vn = V + (size_t)(j + 1) * nv;
    dgemv_dev(N, nrhs, A, lda, Vj, Wv, part, st);                 // A v_j
    ATLB_CUDA_CHECK(cudaMemsetAsync(Z, 0, sizeof(double) * nv, st));
    correct(Wv, N, Z, N);                                          // M^-1 A v_j
    multidot_kernel<<<dim3(j + 1, nrhs), 256, 0, st>>>(N, nrhs, V, Z, h1);
    vcombine_kernel<<<vgrid, 256, 0, st>>>(N, nrhs, j + 1, V, h1, -1.0, Z, N);
    multidot_kernel<<<dim3(j + 1, nrhs), 256, 0, st>>>(N, nrhs, V, Z, h2);
    vcombine_kernel<<<vgrid, 256, 0, st>>>(N, nrhs, j + 1, V, h2, -1.0, Z, N);
    multidot_kernel<<<dim3(1, nrhs), 256, 0, st>>>(N, nrhs, Z, Z, nrm);
    vscale_kernel<<<vgrid, 256, 0, st>>>(N, nrhs, Z, nrm, Vn);
    ATLB_CUDA_CHECK(cudaGetLastError());
    ATLB_CUDA_CHECK(cudaMemcpyAsync(hh1, h1, sizeof(double) * (size_t)(j + 1) * nrhs, cudaMemcpyDeviceToHost, st));
    ATLB_CUDA_CHECK(cudaMemcpyAsync(hh2, h2, sizeof(double) * (size_t)(j + 1) * nrhs, cudaMemcpyDeviceToHost, st));
    ATLB_CUDA_CHECK(cudaMemcpyAsync(hnrm, nrm, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
    ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
    bool done = true;
    for (int c = 0; c < nrhs; c++) {
      double *gc = g.data() + (size_t)c * (m + 1), *csc = cs.data() + (size_t)c * m, *snc = sn.data() + (size_t)c * m;
      for (int i = 0; i <= j; i++) Hc(c, i, j) = hh1[(size_t)i * nrhs + c] + hh2[(size_t)i * nrhs + c];
      Hc(c, j + 1, j) = std::sqrt(std::max(hnrm[c], 0.0));
      for (int i = 0; i < j; i++) {  // previous rotations
        const double t = csc[i] * Hc(c, i, j) + snc[i] * Hc(c, i + 1, j);
        Hc(c, i + 1, j) = -snc[i] * Hc(c, i, j) + csc[i] * Hc(c, i + 1, j);
        Hc(c, i, j) = t;
      }
      const double a = Hc(c, j, j), b = Hc(c, j + 1, j), d = std::hypot(a, b);
      csc[j] = d > 0 ? a / d : 1.0;
      snc[j] = d > 0 ? b / d : 0.0;
      Hc(c, j, j) = d;
      Hc(c, j + 1, j) = 0.0;
      gc[j + 1] = -snc[j] * gc[j];
      gc[j] = csc[j] * gc[j];
      if (!(std::fabs(gc[j + 1]) <= KRYLOV_TAU * beta[c]) && std::isfinite(gc[j + 1])) done = false;
    }
    j++;
    if (debug_ir()) fprintf(stderr, "atlas_b200 gmres: step %d residual estimate %.3e\n", j,
                            std::fabs(g[j]) / std::max(beta[0], 1e-300));
    if (done) break;
  }
  // y = H(0:j, 0:j)^-1 g(0:j) per column (upper triangular after the rotations)
  for (int c = 0; c < nrhs; c++) {
    const double *gc = g.data() + (size_t)c * (m + 1);
    for (int i = j - 1; i >= 0; i--) {
      double s = gc[i];
      for (int k = i + 1; k < j; k++) s -= Hc(c, i, k) * hy[(size_t)k * nrhs + c];
      const double dii = Hc(c, i, i);
      hy[(size_t)i * nrhs + c] = (dii != 0.0 && std::isfinite(s)) ? s / dii : 0.0;
    }
  }
  ATLB_CUDA_CHECK(cudaMemcpyAsync(y, hy, sizeof(double) * (size_t)j * nrhs, cudaMemcpyHostToDevice, st));
  vcombine_kernel<<<vgrid, 256, 0, st>>>(N, nrhs, j, V, y, 1.0, X, ldx);
  ATLB_CUDA_CHECK(cudaGetLastError());
  return j;
}

// Refinement driver shared by the solvers.  `factor(part, nrm)` factors the
// low precision copy and returns its info; it also leaves ||A||_inf (bits of
// the double) in *nrm, with part (N * ceil(N/256) doubles) as workspace, so
// that the copy and the norm can share one pass over A (d2s_norm_dev);
// `correct(R, ldr, X, ldx)` adds an
// approximate solution of A D = R to X (R, X FP64 device); `fallback()` runs
// the FP64 solver.  X is overwritten with the solution.
//
// krylov: 0 = plain refinement only; 1 = plain refinement, switching to
// GMRES-IR corrections (gmres_correct) once a step fails to halve the
// backward error (a plain step and a GMRES step cost about the same -- one
// product with A, one solve with the factors -- so plain steps are kept
// while they converge); 2 = GMRES-IR corrections from the first step.
// GMRES-IR serves up to KRYLOV_MAX_RHS right-hand sides and gives up (FP64
// fallback) after a correction that fails to halve the backward error, or
// after KRYLOV_OUTER of them.
thread_local int tl_krylov_steps = 0;
constexpr int KRYLOV_OUTER = 12;

// the refinement mode for a factorization precision: the tunable, with its
// automatic setting (1) taking GMRES-IR from the start for BF16 factors, whose
// u * kappa * growth is near 1 already for well-conditioned matrices
int krylov_mode(int prec) {
  const int k = tune(kTuneMixedKrylov);
  return (k == 1 && prec == kPrecBF16) ? 2 : k;
}

template <class Factor, class Correct, class Fallback>
int refine(int N, int nrhs, const double *A, long lda, const double *B, long ldb, double *X,
           long ldx, int *iter, Factor factor, Correct correct, Fallback fallback, cudaStream_t st,
           MixedStats *stats, int krylov) {
  tl_krylov_steps = 0;
  const int nch = cdiv(N, GV_COLS);
  double *R = (double *)scratch(kSlotMixedR, sizeof(double) * (size_t)N * nrhs);
  double *part = (double *)scratch(kSlotMixedD, sizeof(double) * (size_t)nch * N * 8 + 64);
  unsigned long long *red = (unsigned long long *)scratch(kSlotWork2, sizeof(unsigned long long) * (3 * nrhs + 8));
  unsigned long long *hred = (unsigned long long *)pinned(kSlotWork2, sizeof(unsigned long long) * (3 * nrhs + 8));

  int finfo = factor(part, red + 3 * nrhs);  // also leaves ||A||_inf (bits) in red[3 nrhs]
  double anrm = 0.0;
  {
    ATLB_CUDA_CHECK(cudaMemcpyAsync(hred, red + 3 * nrhs, 8, cudaMemcpyDeviceToHost, st));
    ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
    anrm = bits_to_double(hred[0]);
  }
  const double tol = N * std::ldexp(1.0, -53);
  if (finfo == 0) {
    for (int r = 0; r < nrhs; r++)
      ATLB_CUDA_CHECK(cudaMemsetAsync(X + (long)r * ldx, 0, sizeof(double) * N, st));
    correct(B, ldb, X, ldx);  // x0
    bool gm = krylov == 2 && nrhs <= KRYLOV_MAX_RHS;
    int gm_outer = 0, gm_stall = 0;  // GMRES-IR corrections taken / that failed to halve the error
    double prev = INFINITY;
    for (int it = 0; it <= ITERMAX; it++) {
      dresid_dev(N, nrhs, A, lda, X, ldx, B, ldb, R, N, part, red, st);
      ATLB_CUDA_CHECK(cudaMemcpyAsync(hred, red, sizeof(unsigned long long) * 3 * nrhs,
                                      cudaMemcpyDeviceToHost, st));
      ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
      bool ok = true;
      double worst = 0.0;
      for (int r = 0; r < nrhs; r++) {
        double rn = bits_to_double(hred[3 * r]), xn = bits_to_double(hred[3 * r + 1]),
               bn = bits_to_double(hred[3 * r + 2]);
        double den = anrm * xn + bn;
        double eta = den > 0 ? rn / den : rn;
        if (!(eta <= tol)) ok = false;
        worst = std::max(worst, std::isfinite(eta) ? eta : 1e300);
      }
      if (stats) { stats->bwd_err = worst; stats->anrm = anrm; }
      if (debug_ir()) fprintf(stderr, "atlas_b200 refine: iter %d backward error %.3e (target %.3e)\n", it, worst, tol);
      if (ok) {
        *iter = it;
        return 0;
      }
      if (it == ITERMAX || !(worst < 1e300)) break;
      if (!gm && krylov == 1 && nrhs <= KRYLOV_MAX_RHS && it >= 1 && !(worst <= 0.5 * prev)) gm = true;
      if (gm && gm_outer > 0 && !(worst <= 0.5 * prev)) gm_stall++;
      if (gm && (gm_stall >= 1 || gm_outer >= KRYLOV_OUTER)) break;
      prev = worst;
      if (gm) {
        tl_krylov_steps += gmres_correct(N, nrhs, A, lda, R, N, X, ldx, correct, part, st);
        gm_outer++;
      } else {
        correct(R, N, X, ldx);
      }
    }
    *iter = -(ITERMAX + 1);
  } else {
    *iter = -3;  // the low-precision factorization broke down (LAPACK dsgesv: ITER = -3)
  }
  return fallback();
}

}  // namespace atlb

using namespace atlb;

namespace {
int read_info(const int *dinfo, cudaStream_t st) {
  int *h = (int *)pinned(kSlotInfo, 64);
  ATLB_CUDA_CHECK(cudaMemcpyAsync(h, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  return *h;
}
}  // namespace

extern "C" {

int atlb_dsgesv_ex(int N, int NRHS, double *A, int lda, int *ipiv, double *B, int ldb, double *X,
                   int ldx, int prec, int pivoting, int *iter) {
  if (N < 0) return -1;
  if (NRHS < 0) return -2;
  if (lda < std::max(1, N)) return -4;
  if (ldb < std::max(1, N)) return -7;
  if (ldx < std::max(1, N)) return -9;
  if (prec < kPrecFP32 || prec > kPrecTF32x3) return -10;
  if (pivoting != 0 && pivoting != 1) return -11;
  int it_local = 0;
  if (!iter) iter = &it_local;
  *iter = 0;
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  // a host A at a size where the copy is long is factored while its second
  // half arrives
  const bool streamed = !pivoting && N >= 2048 && !is_dev(A);
  DMat<double> dA = stage_in(kSlotA, (const double *)A, N, N, lda, !streamed, st);
  DMat<double> dB = stage_in(kSlotB, (const double *)B, N, NRHS, ldb, true, st);
  DMat<double> dX = stage_in(kSlotC, (const double *)X, N, NRHS, ldx, false, st);
  int *dip = stage_vec_in<int>(kSlotIpiv, ipiv, N, false, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  SgemmFn g = factor_gemm(prec);
  bool copied = !streamed;  // the FP64 A is on the device
  const int n4 = rbt_order(N);
  const long lds = pivoting ? n4 : N;
  float *S = (float *)scratch(kSlotMixedA, sizeof(float) * (size_t)lds * lds);
  float *Rs = (float *)scratch(kSlotMixedX, sizeof(float) * (size_t)lds * NRHS);
  double *rd = pivoting ? (double *)scratch(kSlotTc1, sizeof(double) * 4 * n4) : nullptr;
  // few right-hand sides: the solves reuse the factors' inverted diagonal
  // blocks and the net row permutation, computed once after the factorization
  const bool few = NRHS <= 8;
  const int nw = few ? (int)lds : 0;
  float *WL = few ? (float *)scratch(kSlotMixedWL, sizeof(float) * trsv_w_elems(nw)) : nullptr;
  float *WU = few ? (float *)scratch(kSlotMixedWU, sizeof(float) * trsv_w_elems(nw)) : nullptr;
  int *perm = (few && !pivoting) ? (int *)scratch(kSlotMixedPerm, sizeof(int) * (size_t)N) : nullptr;
  auto factor = [&](double *part, unsigned long long *nrm) {
    if (pivoting) {
      dnorm_inf_dev(N, dA.d, dA.ld, part, nrm, st);
      rbt_init_dev(n4, rd, st);
      rbt_matrix_dev(N, dA.d, dA.ld, rd, S, st);
      getrf_nopiv_dev<float>(n4, S, lds, dinfo, st, g);
    } else if (!copied) {
      streamed_factor_dev(N, (const double *)A, lda, dA.d, dA.ld, S, lds, dip, dinfo, part, nrm, g, st);
      copied = true;
      if (few) ipiv_to_perm_dev(N, dip, perm, st);
    } else {
      d2s_norm_dev(N, dA.d, dA.ld, S, lds, part, nrm, st);
      getrf_dev<float>(N, N, S, lds, dip, dinfo, st, g);
      if (few) ipiv_to_perm_dev(N, dip, perm, st);
    }
    if (few) {
      trsv_inverse_dev<float>(kLower, kNoTrans, kUnit, nw, S, lds, WL, st);
      trsv_inverse_dev<float>(kUpper, kNoTrans, kNonUnit, nw, S, lds, WU, st);
    }
    return read_info(dinfo, st);
  };
  auto correct = [&](const double *R, long ldr, double *Xc, long ldxc) {
    if (pivoting) {
      rbt_left_vec_dev(N, NRHS, R, ldr, rd, Rs, st);
      if (few) {
        trsv_w_dev<float>(kLower, kNoTrans, n4, NRHS, S, lds, WL, Rs, n4, st);
        trsv_w_dev<float>(kUpper, kNoTrans, n4, NRHS, S, lds, WU, Rs, n4, st);
      } else {
        trsm_dev<float>(kLeft, kLower, kNoTrans, kUnit, n4, NRHS, 1.f, S, lds, Rs, n4, st, g);
        trsm_dev<float>(kLeft, kUpper, kNoTrans, kNonUnit, n4, NRHS, 1.f, S, lds, Rs, n4, st, g);
      }
      rbt_right_add_dev(N, NRHS, Rs, rd, Xc, ldxc, st);
    } else if (few) {
      gather_d2s_dev(N, NRHS, R, ldr, perm, Rs, N, st);
      trsv_w_dev<float>(kLower, kNoTrans, N, NRHS, S, lds, WL, Rs, N, st);
      trsv_w_dev<float>(kUpper, kNoTrans, N, NRHS, S, lds, WU, Rs, N, st);
      add_s2d_dev(N, NRHS, Rs, N, Xc, ldxc, st);
    } else {
      d2s_dev(N, NRHS, R, ldr, Rs, N, st);
      getrs_dev<float>(kNoTrans, N, NRHS, S, lds, dip, Rs, N, st, g);
      add_s2d_dev(N, NRHS, Rs, N, Xc, ldxc, st);
    }
  };
  bool fell_back = false;
  auto fallback = [&]() {
    // FP64 dgesv on A itself (LAPACK dsgesv: A then holds the FP64 factors)
    fell_back = true;
    getrf_dev<double>(N, N, dA.d, dA.ld, dip, dinfo, st);
    int info = read_info(dinfo, st);
    if (info == 0) {
      for (int r = 0; r < NRHS; r++)
        ATLB_CUDA_CHECK(cudaMemcpyAsync(dX.d + (long)r * dX.ld, dB.d + (long)r * dB.ld,
                                        sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      getrs_dev<double>(kNoTrans, N, NRHS, dA.d, dA.ld, dip, dX.d, dX.ld, st);
    }
    return info;
  };
  int info = refine(N, NRHS, dA.d, dA.ld, dB.d, dB.ld, dX.d, dX.ld, iter, factor, correct, fallback,
                    st, nullptr, krylov_mode(prec));
  stage_out(X, ldx, dX, N, NRHS, st);
  if (fell_back) {
    stage_out(A, lda, dA, N, N, st);
    stage_vec_out<int>(ipiv, dip, N, st);
  }
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  return info;
}

int atlb_mixed_krylov_steps(void) { return tl_krylov_steps; }

int atlb_dsgesv(int N, int NRHS, double *A, int lda, int *ipiv, double *B, int ldb, double *X,
                int ldx, int prec, int *iter) {
  return atlb_dsgesv_ex(N, NRHS, A, lda, ipiv, B, ldb, X, ldx, prec, 0, iter);
}

int atlb_dsposv(int Uplo, int N, int NRHS, double *A, int lda, double *B, int ldb, double *X,
                int ldx, int prec, int *iter) {
  if (Uplo != kUpper && Uplo != kLower) return -1;
  if (N < 0) return -2;
  if (NRHS < 0) return -3;
  if (lda < std::max(1, N)) return -5;
  if (ldb < std::max(1, N)) return -7;
  if (ldx < std::max(1, N)) return -9;
  if (prec < kPrecFP32 || prec > kPrecTF32x3) return -10;
  int it_local = 0;
  if (!iter) iter = &it_local;
  *iter = 0;
  if (N == 0 || NRHS == 0) return 0;
  cudaStream_t st = stream();
  DMat<double> dA = stage_in(kSlotA, (const double *)A, N, N, lda, true, st);
  DMat<double> dB = stage_in(kSlotB, (const double *)B, N, NRHS, ldb, true, st);
  DMat<double> dX = stage_in(kSlotC, (const double *)X, N, NRHS, ldx, false, st);
  int *dinfo = (int *)scratch(kSlotInfo, 64);
  SgemmFn g = factor_gemm(prec);
  // The residual needs all of A: the other triangle is taken from the
  // referenced one by symmetry (a full symmetric copy, FP64).
  double *Af = (double *)scratch(kSlotWork, sizeof(double) * (size_t)N * N);
  symmetrize_dev(Uplo, N, dA.d, dA.ld, Af, N, st);
  float *S = (float *)scratch(kSlotMixedA, sizeof(float) * (size_t)N * N);
  float *Rs = (float *)scratch(kSlotMixedX, sizeof(float) * (size_t)N * NRHS);
  const bool few = NRHS <= 8;
  float *W1 = few ? (float *)scratch(kSlotMixedWL, sizeof(float) * trsv_w_elems(N)) : nullptr;
  float *W2 = few ? (float *)scratch(kSlotMixedWU, sizeof(float) * trsv_w_elems(N)) : nullptr;
  // A = L L^T (or U^T U): the factor mirrored into the other triangle of S,
  // then a lower solve with L (or U^T) and an upper one with L^T (or U), both
  // reading S column by column
  auto factor = [&](double *part, unsigned long long *nrm) {
    d2s_norm_dev(N, Af, N, S, N, part, nrm, st);
    potrf_dev<float>(Uplo, N, S, N, dinfo, st, g);
    if (few) {
      const dim3 tiles(cdiv(N, 32), cdiv(N, 32));
      mirror_tri_kernel<<<tiles, dim3(32, 8), 0, st>>>(Uplo, N, S, N);
      ATLB_CUDA_CHECK(cudaGetLastError());
      trsv_inverse_dev<float>(kLower, kNoTrans, kNonUnit, N, S, N, W1, st);
      trsv_inverse_dev<float>(kUpper, kNoTrans, kNonUnit, N, S, N, W2, st);
    }
    return read_info(dinfo, st);
  };
  auto correct = [&](const double *R, long ldr, double *Xc, long ldxc) {
    d2s_dev(N, NRHS, R, ldr, Rs, N, st);
    if (few) {
      trsv_w_dev<float>(kLower, kNoTrans, N, NRHS, S, N, W1, Rs, N, st);
      trsv_w_dev<float>(kUpper, kNoTrans, N, NRHS, S, N, W2, Rs, N, st);
    } else {
      potrs_dev<float>(Uplo, N, NRHS, S, N, Rs, N, st, g);
    }
    add_s2d_dev(N, NRHS, Rs, N, Xc, ldxc, st);
  };
  bool fell_back = false;
  auto fallback = [&]() {
    fell_back = true;
    potrf_dev<double>(Uplo, N, dA.d, dA.ld, dinfo, st);
    int info = read_info(dinfo, st);
    if (info == 0) {
      for (int r = 0; r < NRHS; r++)
        ATLB_CUDA_CHECK(cudaMemcpyAsync(dX.d + (long)r * dX.ld, dB.d + (long)r * dB.ld,
                                        sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      potrs_dev<double>(Uplo, N, NRHS, dA.d, dA.ld, dX.d, dX.ld, st);
    }
    return info;
  };
  int info = refine(N, NRHS, Af, N, dB.d, dB.ld, dX.d, dX.ld, iter, factor, correct, fallback, st,
                    nullptr, krylov_mode(prec));
  stage_out(X, ldx, dX, N, NRHS, st);
  if (fell_back) stage_out(A, lda, dA, N, N, st);
  ATLB_CUDA_CHECK(cudaStreamSynchronize(st));
  return info;
}

}  // extern "C"
