// Interface of the tcgen05 GEMM (tc_gemm.cu) shared with its users.
#pragma once
#include <cuda_runtime.h>

namespace atlb {
namespace tc {

enum { kKindBF16 = 0, kKindTF32 = 1, kKindI8 = 2 };
enum { kEpiF32 = 0, kEpiF64Acc = 1 };

struct EpiParams {
  float *Cf;         // kEpiF32: C = alpha*D + beta*C (column-major, ldc)
  double *Cd;        // kEpiF64Acc: C += w * rs[m] * cs[n] * D
  long ldc;
  float alpha, beta;
  int tri;           // kEpiF32 only: 0 all, 1 lower (m >= n), 2 upper
  double w;
  const double *rs, *cs;
};

// D = A * B^T with A (M x K) and B (N x K) K-major (leading dimensions in
// elements, 16-byte aligned rows); the epilogue consumes D.
void tc_gemm(int kind, int epi, const void *A, long lda, const void *B, long ldb, int M, int N,
             int K, const EpiParams &ep, cudaStream_t st);
// Error code recorded by a kernel whose bounded wait timed out (0 = none);
// reading it synchronises the stream and clears it.
int read_and_clear_error(cudaStream_t st);

}  // namespace tc
}  // namespace atlb
