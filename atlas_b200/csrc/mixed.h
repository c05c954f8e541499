// Mixed-precision building blocks (mixed.cu) shared with the C ABI layer.
#pragma once
#include <cstring>
#include <cuda_runtime.h>
#include "kernels.h"

namespace atlb {

enum { kPrecFP32 = 0, kPrecTF32 = 1, kPrecBF16 = 2, kPrecTF32x3 = 3 };

struct MixedStats {
  double bwd_err;  // worst normwise backward error at exit
  double anrm;     // ||A||_inf
};

inline double bits_to_double(unsigned long long u) {
  double d;
  std::memcpy(&d, &u, sizeof d);
  return d;
}

SgemmFn factor_gemm(int prec);
int rbt_order(int n);
void rbt_init_dev(int n4, double *d, cudaStream_t st);
void rbt_matrix_dev(int n, const double *A, long lda, const double *d, float *S, cudaStream_t st);
void rbt_left_vec_dev(int n, int nrhs, const double *R, long ldr, const double *d, float *C,
                      cudaStream_t st);
void rbt_right_add_dev(int n, int nrhs, const float *Y, const double *d, double *X, long ldx,
                       cudaStream_t st);
void symmetrize_dev(int uplo, int N, const double *A, long lda, double *F, long ldf, cudaStream_t st);
void dnorm_inf_dev(int N, const double *A, long lda, double *part, unsigned long long *out,
                   cudaStream_t st);
void dresid_dev(int N, int nrhs, const double *A, long lda, const double *X, long ldx,
                const double *B, long ldb, double *R, long ldr, double *part,
                unsigned long long *red, cudaStream_t st);
void d2s_dev(int M, int N, const double *A, long lda, float *S, long lds, cudaStream_t st);
void s2d_dev(int M, int N, const float *S, long lds, double *X, long ldx, cudaStream_t st);
void add_s2d_dev(int M, int N, const float *S, long lds, double *X, long ldx, cudaStream_t st);

}  // namespace atlb
