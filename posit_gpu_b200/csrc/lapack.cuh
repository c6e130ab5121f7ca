// lapack.cuh -- device-resident posit32 factorizations and solves (lapack.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pg {

// The measured-best panel width for an n x n LU (lu) or lower Cholesky factorization.
int tuned_panel_width(bool lu, int n);
size_t rgetrf_workspace_bytes(int m, int n, int nb);
size_t rpotrf_workspace_bytes(int n, int nb);

// All pointers are device pointers; ipiv is 1-based as in the reference; *info must be
// zero on entry (it receives the first zero pivot / the first non-positive diagonal).
// max_ctas caps the thread-block cluster of a panel held in shared memory (0: up to 8); a
// caller that runs many factorizations at once uses smaller clusters, which the GPU can
// place beside other work.  The bits do not depend on it.
cudaError_t rgetrf_launch(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info, void *ws,
                          cudaStream_t st, int max_ctas = 0);
cudaError_t rpotrf_lower_launch(int n, uint32_t *A, int lda, int nb, int *info, void *ws, cudaStream_t st,
                                int max_ctas = 0);
cudaError_t rgetrs_launch(int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb,
                          cudaStream_t st);
cudaError_t rpotrs_lower_launch(int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb,
                                cudaStream_t st);
// Upper Cholesky (nb-dependent bits: the caller's nb is the reference's), its solve, and
// the transposed LU solve.
size_t rpotrf_upper_workspace_bytes(int n, int nb);
cudaError_t rpotrf_upper_launch(int n, uint32_t *A, int lda, int nb, int *info, void *ws, cudaStream_t st);
cudaError_t rpotrs_upper_launch(int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb,
                                cudaStream_t st);
cudaError_t rgetrs_trans_launch(int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb,
                                cudaStream_t st);

} // namespace pg
