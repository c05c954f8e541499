// Device-pointer building blocks shared by the drivers and the C-ABI layer.
// All routines are column-major, enqueue on `st` and return without waiting.
#pragma once
#include <cuda_runtime.h>

namespace atlb {

// C = alpha*op(A)*op(B) + beta*C.  tri: 0 whole C, 1 lower triangle only,
// 2 upper triangle only (SYRK).
void dgemm_dev(int ta, int tb, int M, int N, int K, double alpha, const double *A, long lda,
               const double *B, long ldb, double beta, double *C, long ldc, cudaStream_t st,
               int tri = 0);
void sgemm_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
               const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
               int tri = 0);

// One problem of a grouped (batched, uneven) DGEMM: C = alpha*op(A)*op(B) + beta*C.
struct GemmProb {
  const double *A, *B;
  double *C;
  int M, N, K;
  long lda, ldb, ldc;
  double alpha, beta;
};
// All problems share TransA / TransB; device pointers; one persistent launch.
void dgemm_grouped_dev(int ta, int tb, const GemmProb *hprobs, int count, cudaStream_t st);

// A FP32 GEMM entry with the sgemm_dev signature; the mixed-precision LU and
// Cholesky take one of these for their trailing updates.
typedef void (*SgemmFn)(int ta, int tb, int M, int N, int K, float alpha, const float *A,
                        long lda, const float *B, long ldb, float beta, float *C, long ldc,
                        cudaStream_t st, int tri);

// Tensor-core (tcgen05) FP32-in/FP32-out GEMMs: operands rounded to TF32 or
// BF16 on the fly, FP32 accumulation in tensor memory.
void sgemm_tf32_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                    const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                    int tri);
void sgemm_bf16_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                    const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                    int tri);
// Near-FP32 GEMM on the TF32 tensor cores (operands split into TF32 high and
// low planes, three products per k-step into one accumulator).
void sgemm_tf32x3_dev(int ta, int tb, int M, int N, int K, float alpha, const float *A, long lda,
                      const float *B, long ldb, float beta, float *C, long ldc, cudaStream_t st,
                      int tri);

template <typename T>
void gemm_dev(int ta, int tb, int M, int N, int K, T alpha, const T *A, long lda, const T *B,
              long ldb, T beta, T *C, long ldc, cudaStream_t st, int tri = 0);

// Triangular solve (BLAS trsm semantics), recursive with GEMM off-diagonal
// updates; `gemm` is used for the FP32 instantiation (nullptr = sgemm_dev).
template <typename T>
void trsm_dev(int side, int uplo, int trans, int diag, int M, int N, T alpha, const T *A, long lda,
              T *B, long ldb, cudaStream_t st, SgemmFn gemm = nullptr);
// B = L^-1 B for L unit lower triangular of order m <= 256 (left, lower,
// no transpose, unit diagonal) in one launch.
template <typename T>
void trsm_llu_small_dev(int m, int n, const T *L, long lda, T *B, long ldb, cudaStream_t st);
// The TRSM with its workspace supplied: W holds ceil(n/64) blocks of 64x64
// elements (n = order of the triangle).
template <typename T>
void trsm_impl(int side, int uplo, int trans, int diag, int M, int N, T alpha, const T *A, long lda,
               T *B, long ldb, cudaStream_t st, SgemmFn gemm, T *W);
// Inverses of the 64x64 diagonal blocks of the triangle T(i,k) = Tp[i*tr + k*tc]
// (n x n), block b stored dense 64x64 column-major at W + b*4096.
template <typename T>
void trinv_dev(int n, const T *Tp, long tr, long tc, int lower, int unit, T *W, cudaStream_t st);
// op(A) X = B (Left side): one launch per 8 right-hand sides, the inverted
// diagonal blocks computed once.  getrs / potrs take this path up to
// kTrsvMaxRhs right-hand sides, the recursive TRSM above.
constexpr int kTrsvMaxRhs = 32;
template <typename T>
void trsv_dev(int uplo, int trans, int diag, int n, int nrhs, const T *A, long lda, T *B, long ldb,
              cudaStream_t st);
// W for trsv_w_dev: the inverted 128 x 128 diagonal blocks (W holds trsv_w_elems(n) elements)
size_t trsv_w_elems(int n);
template <typename T>
void trsv_inverse_dev(int uplo, int trans, int diag, int n, const T *A, long lda, T *W, cudaStream_t st);
template <typename T>
void trsv_w_dev(int uplo, int trans, int n, int nrhs, const T *A, long lda, const T *W, T *B, long ldb,
                cudaStream_t st);
// net row permutation of ipiv[0..n) applied forward: row i of P*B is row perm[i] of B
void ipiv_to_perm_dev(int n, const int *ipiv, int *perm, cudaStream_t st);
// depth-one look-ahead in the blocked factorizations (ATLAS_B200_LOOKAHEAD=0 turns it off)
bool lookahead_enabled();

// B = alpha*op(A)*B (Left) or alpha*B*op(A) (Right), A triangular.
void dtrmm_dev(int side, int uplo, int trans, int diag, int M, int N, double alpha,
               const double *A, long lda, double *B, long ldb, cudaStream_t st);

// Row interchanges: for k = k1..k2-1 (inc > 0) or k2-1..k1 (inc < 0) swap
// rows k and ipiv[k] of the ncols columns starting at A (row indices are
// absolute: row r of the matrix is A[r]).
template <typename T>
void laswp_dev(int ncols, T *A, long lda, int k1, int k2, const int *ipiv, int inc,
               cudaStream_t st);

// LU with partial pivoting, ATLAS's recursive splitting.  ipiv: device,
// 0-based absolute rows.  dinfo: device int, receives 0 or the first zero
// pivot (1-based).
template <typename T>
void getrf_dev(int M, int N, T *A, long lda, int *ipiv, int *dinfo, cudaStream_t st,
               SgemmFn gemm = nullptr);
// LU without pivoting (for matrices made pivot-safe by a random butterfly
// transformation); dinfo as above.
template <typename T>
void getrf_nopiv_dev(int N, T *A, long lda, int *dinfo, cudaStream_t st, SgemmFn gemm = nullptr);
template <typename T>
void getrs_dev(int trans, int N, int NRHS, const T *A, long lda, const int *ipiv, T *B, long ldb,
               cudaStream_t st, SgemmFn gemm = nullptr);

// Cholesky (uplo = kLower: A = L L^T; kUpper: A = U^T U); dinfo as above.
template <typename T>
void potrf_dev(int uplo, int N, T *A, long lda, int *dinfo, cudaStream_t st,
               SgemmFn gemm = nullptr);
template <typename T>
void potrs_dev(int uplo, int N, int NRHS, const T *A, long lda, T *B, long ldb, cudaStream_t st,
               SgemmFn gemm = nullptr);

// Householder QR (ATLAS conventions: tau in [1,2], beta = -sign(alpha)*norm).
void dgeqrf_dev(int M, int N, double *A, long lda, double *tau, cudaStream_t st);
// C = op(Q) C (side kLeft, Q of order M) or C op(Q) (kRight, order N), Q from
// dgeqrf_dev's K reflectors in A and tau (ATL_ormqr).
void dormqr_dev(int side, int trans, int M, int N, int K, const double *A, long lda, const double *tau,
                double *C, long ldc, cudaStream_t st);
// D (cols x rows) = S^T
void transpose_dev(int rows, int cols, const double *S, long lds, double *D, long ldd, cudaStream_t st);
// F = A with the triangle `uplo` mirrored into the other one (full symmetric copy)
void symmetrize_dev(int uplo, int N, const double *A, long lda, double *F, long ldf, cudaStream_t st);

// Small utilities
void set_info_kernel_launch(int *dinfo, cudaStream_t st);       // *dinfo = INT_MAX
void finish_info_kernel_launch(int *dinfo, cudaStream_t st);    // INT_MAX -> 0
template <typename T>
void fill_zero_dev(T *A, int M, int N, long lda, cudaStream_t st);

}  // namespace atlb
