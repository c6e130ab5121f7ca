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

// The per-element steps are the FP64 form of p32_mul + p32_add (posit32.cuh,
// f64_posit_mac_checked): operands converted from patterns, the result assembled back
// without rounding.  Row k and column k of a factor step are staged in shared memory as
// FP64 when 2n doubles fit in the staging buffer.
constexpr int STAGE_DOUBLES = BATCH_MAX_N / 2; // s_row (BATCH_MAX_N words) as FP64

__device__ __forceinline__ double pd(uint32_t u) { return p32_to_double(u); }

// b <- b + t*a on patterns through the FP64 step
__device__ __forceinline__ void mac_store(uint32_t *p, double t, double a)
{
    *p = p32_from_double_exact(f64_posit_mac_checked(pd(*p), t, a));
}

// Walks the rows x rows trailing block of step k as flat indexes e = tid, tid + BT, ...
// (row fastest) without a division per element.
struct TrailWalk {
    int i, c;           // the current element (row, column)
    int di, dc, lo, hi; // the step, and the row range [lo, hi)
    __device__ TrailWalk(int rows, int k)
        : i(k + 1 + (int)threadIdx.x % rows), c(k + 1 + (int)threadIdx.x / rows), di(BT % rows), dc(BT / rows),
          lo(k + 1), hi(k + 1 + rows)
    {
    }
    __device__ void next()
    {
        i += di;
        c += dc;
        if (i >= hi) {
            i -= hi - lo;
            ++c;
        }
    }
};

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
                s_recip = pdiv_est(P32_ONE, piv);
            } else {
                s_mode = 2;
            }
            s_piv = piv;
        }
        if (piv == 0 && info == 0)
            info = k + 1;
        __syncthreads();
        if (p != k) { // interchange whole rows (Rlaswp on both sides)
            // A zero pivot leaves its own column in place (Rgetrf2.cpp:107-117) while the
            // recursion's Rlaswp calls still move rows k and p in every other column.
            for (int c = tid; c < n; c += blockDim.x) {
                if (c == k && piv == 0)
                    continue;
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
                l = pdiv_est(l, s_piv);
            ck[i] = l;
        }
        const bool stage = 2 * n <= STAGE_DOUBLES;
        double *s_rowd = reinterpret_cast<double *>(s_row), *s_cold = s_rowd + n;
        for (int c = k + 1 + tid; c < n; c += blockDim.x) {
            const uint32_t v = pneg(A[k + (size_t)c * lda]);
            if (stage)
                s_rowd[c] = pd(v);
            else
                s_row[c] = v;
        }
        if (stage)
            for (int i = k + 1 + tid; i < n; i += blockDim.x)
                s_cold[i] = pd(ck[i]);
        __syncthreads();
        const int rows = n - k - 1;
        if (rows > 0) {
            TrailWalk w(rows, k);
            for (; w.c < n; w.next()) {
                const double t = stage ? s_rowd[w.c] : pd(s_row[w.c]);
                const double l = stage ? s_cold[w.i] : pd(ck[w.i]);
                mac_store(A + w.i + (size_t)w.c * lda, t, l);
            }
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
                mac_store(b + i, -pd(bk), pd(lk[i]));
        }
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        const uint32_t *uk = A + (size_t)k * lda;
        for (int r = tid; r < nrhs; r += blockDim.x) {
            uint32_t *b = pr.B + (size_t)r * ldb;
            if (b[k] != 0)
                b[k] = pdiv_est(b[k], uk[k]);
        }
        __syncthreads();
        for (int e = tid; e < k * nrhs; e += blockDim.x) {
            uint32_t *b = pr.B + (size_t)(e / k) * ldb;
            const int i = e % k;
            const uint32_t bk = b[k];
            if (bk != 0)
                mac_store(b + i, -pd(bk), pd(uk[i]));
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
                uint32_t lkk = psqrt_est(akk);
                ck[k] = lkk;
                s_recip = pdiv_est(P32_ONE, lkk);
            }
        }
        __syncthreads();
        if (s_fail) {
            info = k + 1;
            break;
        }
        const bool stage = n <= STAGE_DOUBLES;
        double *s_cold = reinterpret_cast<double *>(s_row);
        for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            const uint32_t l = pmul(s_recip, ck[i]);
            ck[i] = l;
            if (stage)
                s_cold[i] = pd(l);
            else
                s_row[i] = l;
        }
        __syncthreads();
        // lower part of the trailing matrix: a_ic += (-l_ck)*l_ik, k < c <= i
        const int rows = n - k - 1;
        if (rows > 0) {
            TrailWalk w(rows, k);
            for (; w.c < n; w.next()) {
                if (w.i >= w.c) {
                    const double lc = stage ? s_cold[w.c] : pd(s_row[w.c]);
                    const double li = stage ? s_cold[w.i] : pd(s_row[w.i]);
                    mac_store(A + w.i + (size_t)w.c * lda, -lc, li);
                }
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
                b[k] = pdiv_est(b[k], lk[k]);
        }
        __syncthreads();
        const int rows = n - k - 1;
        for (int e = tid; e < rows * nrhs; e += blockDim.x) {
            uint32_t *b = pr.B + (size_t)(e / rows) * ldb;
            const int i = k + 1 + e % rows;
            const uint32_t bk = b[k];
            if (bk != 0)
                mac_store(b + i, -pd(bk), pd(lk[i]));
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

#ifndef PG_BATCH_MIN_CTAS
#define PG_BATCH_MIN_CTAS 6 // 40 registers: 6 resident CTAs per SM (measured best of 2, 3, 4, 6, 8)
#endif
__global__ void __launch_bounds__(BT, PG_BATCH_MIN_CTAS) batch_factor_kernel(const BatchProblem *__restrict__ probs, int nprob,
                                                          const int *__restrict__ order, int *__restrict__ next)
{
    __shared__ int32_t s_key[BT];
    __shared__ int s_idx[BT];
    __shared__ int s_item;
    __shared__ __align__(16) uint32_t s_row[BATCH_MAX_N]; // also staged FP64 (8-byte aligned)
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
