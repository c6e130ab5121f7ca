// batch.cuh -- batched posit32 factor-and-solve problems (batch.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pg {

constexpr int BATCH_LU = 0;
constexpr int BATCH_CHOL = 1;
constexpr int BATCH_MAX_N = 4096; // largest n a batched problem may have

// One problem: A (n x n, column-major, lda) is factored in place, B (n x nrhs, ldb)
// overwritten with the solution; ipiv (LU) receives n 1-based pivots, info the
// reference's info.  All pointers are device pointers.
constexpr int BATCH_SOLVE_ONLY = 2; // flag added to kind: A (and ipiv) already factored

struct BatchProblem {
    int kind; // BATCH_LU or BATCH_CHOL, plus BATCH_SOLVE_ONLY
    int n, lda, nrhs, ldb;
    uint32_t *A;
    uint32_t *B;
    int *ipiv;
    int *info;
};

// Runs problems probs[order[i]] (order may be null) on `ctas` persistent CTAs; `next`
// is a device counter the launch zeroes first.
cudaError_t batch_factor_launch(const BatchProblem *probs, int nprob, const int *order, int *next, int ctas,
                                cudaStream_t st);

} // namespace pg
