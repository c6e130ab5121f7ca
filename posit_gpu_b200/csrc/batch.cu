// batch.cu -- many independent posit32 LU / Cholesky factor-and-solve problems in one
// persistent launch fed by a device work queue.
//
// Each CTA takes the next problem from the queue (an atomic counter over a list sorted by
// decreasing size, so the largest problems start first) and factors and solves it alone:
// right-looking, one column per step, the matrix and right-hand sides in global memory
// (L2-resident for the sizes batched here).  Per-element operation order is the
// reference's (see lapack.cu), so every factor, pivot and solution is bit-identical to
// the per-call path (posit_rgetrf_dev + posit_rgetrs_dev, posit_rpotrf_dev +
// posit_rpotrs_dev) and to the CPU routines.
#include "batch.cuh"
#include "posit32.cuh"
#include "trsm_chain.cuh"

namespace pg {

namespace {

constexpr int BT = 256; // threads per problem

__device__ int iramax_block(const uint32_t *col, int k, int n, int32_t *s_key, int *s_idx)
{
    const int tid = threadIdx.x;
    int32_t best = INT32_MIN;
    int bidx = -1;
    for (int i = k + tid; i < n; i += blockDim.x) {
        int32_t key = (int32_t)pabs(col[i]);
        if (bidx < 0 || key > best) {
            best = key;
            bidx = i;
        }
    }
    s_key[tid] = best;
    s_idx[tid] = bidx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) {
            int32_t k2 = s_key[tid + s];
            int i2 = s_idx[tid + s];
            if (i2 >= 0 && (s_idx[tid] < 0 || k2 > s_key[tid] || (k2 == s_key[tid] && i2 < s_idx[tid]))) {
                s_key[tid] = k2;
                s_idx[tid] = i2;
            }
        }
        __syncthreads();
    }
    int p = s_idx[0];
    __syncthreads();
    return p;
}

// Rgetrf (as unblocked right-looking LU) + Rgetrs('N') for one problem.
__device__ void lu_solve_one(const BatchProblem &pr, bool factor, int32_t *s_key, int *s_idx, uint32_t *s_row)
{
    const int n = pr.n, tid = threadIdx.x;
    uint32_t *A = pr.A;
    const size_t lda = (size_t)pr.lda;
    int info = 0;
    __shared__ uint32_t s_piv, s_recip;
    __shared__ int s_mode;
    for (int k = 0; k < (factor ? n : 0); ++k) {
        uint32_t *ck = A + (size_t)k * lda;
        const int p = iramax_block(ck, k, n, s_key, s_idx);
        const uint32_t piv = ck[p];
        if (tid == 0) {
            pr.ipiv[k] = p + 1;
            if (piv == 0) {
                s_mode = 0;
            } else if ((int32_t)pabs(piv) >= 1) {
                s_mode = 1;
                s_recip = pdiv(P32_ONE, piv);
            } else {
                s_mode = 2;
            }
            s_piv = piv;
        }
        if (piv == 0 && info == 0)
            info = k + 1;
        __syncthreads();
        if (piv != 0 && p != k) { // interchange whole rows (Rlaswp on both sides)
            for (int c = tid; c < n; c += blockDim.x) {
                uint32_t *pc = A + (size_t)c * lda;
                uint32_t t = pc[k];
                pc[k] = pc[p];
                pc[p] = t;
            }
        }
        __syncthreads();
        const int mode = s_mode;
        for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            uint32_t l = ck[i];
            if (mode == 1)
                l = pmul(s_recip, l);
            else if (mode == 2)
                l = pdiv(l, s_piv);
            ck[i] = l;
        }
        for (int c = k + 1 + tid; c < n; c += blockDim.x)
            s_row[c] = pneg(A[k + (size_t)c * lda]);
        __syncthreads();
        const int rows = n - k - 1;
        const int cnt = rows * rows;
        for (int e = tid; e < cnt; e += blockDim.x) {
            const int i = k + 1 + e % rows, c = k + 1 + e / rows;
            uint32_t *pc = A + i + (size_t)c * lda;
            *pc = padd(*pc, pmul(s_row[c], ck[i]));
        }
        __syncthreads();
    }
    if (tid == 0 && factor)
        *pr.info = info;
    // Rgetrs 'N': interchanges, L (unit) forward, U backward; the right-hand sides in
    // parallel (each column's per-element order is Rtrsm's, Rtrsm.cpp:121-154)
    const int nrhs = pr.nrhs;
    const size_t ldb = (size_t)pr.ldb;
    for (int r = tid; r < nrhs; r += blockDim.x) { // Rlaswp, in order, on the own column
        uint32_t *b = pr.B + (size_t)r * ldb;
        for (int i = 0; i < n; ++i) {
            const int ip = pr.ipiv[i] - 1;
            if (ip != i) {
                const uint32_t t = b[i];
                b[i] = b[ip];
                b[ip] = t;
            }
        }
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const int rows = n - k - 1;
        const uint32_t *lk = A + (size_t)k * lda;
        for (int e = tid; e < rows * nrhs; e += blockDim.x) {
            uint32_t *b = pr.B + (size_t)(e / rows) * ldb;
            const int i = k + 1 + e % rows;
            const uint32_t bk = b[k];
            if (bk != 0)
                b[i] = padd(b[i], pmul(pneg(bk), lk[i]));
        }
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        const uint32_t *uk = A + (size_t)k * lda;
        for (int r = tid; r < nrhs; r += blockDim.x) {
            uint32_t *b = pr.B + (size_t)r * ldb;
            if (b[k] != 0)
                b[k] = pdiv(b[k], uk[k]);
        }
        __syncthreads();
        for (int e = tid; e < k * nrhs; e += blockDim.x) {
            uint32_t *b = pr.B + (size_t)(e / k) * ldb;
            const int i = e % k;
            const uint32_t bk = b[k];
            if (bk != 0)
                b[i] = padd(b[i], pmul(pneg(bk), uk[i]));
        }
        __syncthreads();
    }
}

// Rpotrf('L') (as unblocked right-looking Cholesky) + Rpotrs('L') for one problem.
__device__ void chol_solve_one(const BatchProblem &pr, bool factor, uint32_t *s_row)
{
    const int n = pr.n, tid = threadIdx.x;
    uint32_t *A = pr.A;
    const size_t lda = (size_t)pr.lda;
    __shared__ uint32_t s_recip;
    __shared__ int s_fail;
    int info = 0;
    for (int k = 0; k < (factor ? n : 0); ++k) {
        uint32_t *ck = A + (size_t)k * lda;
        if (tid == 0) {
            uint32_t akk = ck[k];
            s_fail = (int32_t)akk <= 0;
            if (!s_fail) {
                uint32_t lkk = psqrt(akk);
                ck[k] = lkk;
                s_recip = pdiv(P32_ONE, lkk);
            }
        }
        __syncthreads();
        if (s_fail) {
            info = k + 1;
            break;
        }
        for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            const uint32_t l = pmul(s_recip, ck[i]);
            ck[i] = l;
            s_row[i] = pneg(l);
        }
        __syncthreads();
        // lower part of the trailing matrix: a_ic += (-l_ck)*l_ik, k < c <= i
        const int rows = n - k - 1;
        const int cnt = rows * rows;
        for (int e = tid; e < cnt; e += blockDim.x) {
            const int i = k + 1 + e % rows, c = k + 1 + e / rows;
            if (i >= c) {
                uint32_t *pc = A + i + (size_t)c * lda;
                *pc = padd(*pc, pmul(s_row[c], ck[i]));
            }
        }
        __syncthreads();
    }
    if (tid == 0 && factor)
        *pr.info = info;
    if (info != 0)
        return;
    // Rpotrs 'L': L forward (Rtrsm.cpp:139-154, non-unit), the right-hand sides in
    // parallel; then L^T backward, one thread's chain per right-hand side (trsm_chain.cuh)
    const int nrhs = pr.nrhs;
    const size_t ldb = (size_t)pr.ldb;
    for (int k = 0; k < n; ++k) {
        const uint32_t *lk = A + (size_t)k * lda;
        for (int r = tid; r < nrhs; r += blockDim.x) {
            uint32_t *b = pr.B + (size_t)r * ldb;
            if (b[k] != 0)
                b[k] = pdiv(b[k], lk[k]);
        }
        __syncthreads();
        const int rows = n - k - 1;
        for (int e = tid; e < rows * nrhs; e += blockDim.x) {
            uint32_t *b = pr.B + (size_t)(e / rows) * ldb;
            const int i = k + 1 + e % rows;
            const uint32_t bk = b[k];
            if (bk != 0)
                b[i] = padd(b[i], pmul(pneg(bk), lk[i]));
        }
        __syncthreads();
    }
    // L^T backward: the right-hand sides staged in shared memory when they fit
    const bool staged = n * nrhs <= BATCH_MAX_N;
    if (staged)
        for (int e = tid; e < n * nrhs; e += blockDim.x)
            s_row[e] = pr.B[(size_t)(e / n) * ldb + e % n];
    __syncthreads();
    for (int r = tid; r < nrhs; r += blockDim.x)
        llt_chain(A, lda, staged ? s_row + (size_t)r * n : pr.B + (size_t)r * ldb, n, false);
    __syncthreads();
    if (staged)
        for (int e = tid; e < n * nrhs; e += blockDim.x)
            pr.B[(size_t)(e / n) * ldb + e % n] = s_row[e];
}

} // namespace

__global__ void __launch_bounds__(BT) batch_factor_kernel(const BatchProblem *__restrict__ probs, int nprob,
                                                          const int *__restrict__ order, int *__restrict__ next)
{
    __shared__ int32_t s_key[BT];
    __shared__ int s_idx[BT];
    __shared__ int s_item;
    __shared__ uint32_t s_row[BATCH_MAX_N];
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(next, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= nprob)
            return;
        const BatchProblem pr = probs[order ? order[item] : item];
        const bool factor = !(pr.kind & BATCH_SOLVE_ONLY);
        if ((pr.kind & 1) == BATCH_LU)
            lu_solve_one(pr, factor, s_key, s_idx, s_row);
        else
            chol_solve_one(pr, factor, s_row);
        __syncthreads();
    }
}

cudaError_t batch_factor_launch(const BatchProblem *probs, int nprob, const int *order, int *next, int ctas,
                                cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return e;
    batch_factor_kernel<<<ctas, BT, 0, st>>>(probs, nprob, order, next);
    return cudaGetLastError();
}

} // namespace pg
