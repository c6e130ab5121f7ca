// capi.cu -- the C ABI declared in include/posit_gpu.h.
#include "../../include/posit_gpu.h"
#include "gemm.cuh"
#include "lapack.cuh"
#include "posit32.cuh"

#include <atomic>
#include <ctype.h>
#include <mutex>

namespace {

std::atomic<int> g_last_cuda_error{0};
std::once_flag g_pool_once;

int cuda_fail(cudaError_t e)
{
    g_last_cuda_error.store((int)e);
    if (e == cudaErrorMemoryAllocation)
        return POSIT_E_NO_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return POSIT_E_NO_DEVICE;
    return POSIT_E_CUDA;
}

#define PG_TRY(expr)                                                                                       \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return cuda_fail(e_);                                                                          \
    } while (0)

bool same(char a, char b) { return toupper((unsigned char)a) == toupper((unsigned char)b); }
int imax(int a, int b) { return a > b ? a : b; }

} // namespace

namespace pg {
// Rgemm.cpp:90-128: argument checks in the reference's order.
int rgemm_check_args(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc, bool &nota, bool &notb)
{
    nota = same(ta, 'N');
    notb = same(tb, 'N');
    int nrowa = nota ? m : k, nrowb = notb ? k : n;
    if (!nota && !same(ta, 'C') && !same(ta, 'T'))
        return 1;
    if (!notb && !same(tb, 'C') && !same(tb, 'T'))
        return 2;
    if (m < 0)
        return 3;
    if (n < 0)
        return 4;
    if (k < 0)
        return 5;
    if (lda < imax(1, nrowa))
        return 8;
    if (ldb < imax(1, nrowb))
        return 10;
    if (ldc < imax(1, m))
        return 13;
    return 0;
}
} // namespace pg

namespace {
using pg::rgemm_check_args;

// Keep stream-ordered allocations cached in the device's default pool instead of
// returning them to the driver at every synchronisation.
void init_pool()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
}

int ensure_init()
{
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return e != cudaSuccess ? cuda_fail(e) : POSIT_E_NO_DEVICE;
    std::call_once(g_pool_once, init_pool);
    return 0;
}

// Device-side body shared by both entry points (arguments already checked).
int rgemm_device(bool nota, bool notb, int m, int n, int k, uint32_t alpha, const uint32_t *A, int lda,
                 const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc, void *ws, size_t ws_bytes,
                 cudaStream_t st)
{
    // quick returns and alpha == 0 (Rgemm.cpp:134-157)
    if (m == 0 || n == 0 || ((alpha == 0 || k == 0) && beta == pg::P32_ONE))
        return 0;
    if (alpha == 0 || k == 0) {
        // alpha == 0: C <- 0 or beta*C (Rgemm.cpp:142-156).  k == 0: NN/NT only scale C
        // (Rgemm.cpp:169-177); TN/TT still form alpha*0 and combine it with beta*C
        // (Rgemm.cpp:193-201), NaR when alpha is NaR.
        PG_TRY(pg::scale_launch(m, n, alpha != 0 && !nota, alpha, beta, C, ldc, st));
        return 0;
    }
    size_t need = pg::gemm_workspace_bytes(m, n, k);
    bool own = false;
    if (ws == nullptr) {
        PG_TRY(cudaMallocAsync(&ws, need, st));
        own = true;
    } else if (ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 15u)) {
        return POSIT_E_WORKSPACE;
    }
    cudaError_t e = pg::gemm_launch(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ws, st);
    if (own)
        cudaFreeAsync(ws, st);
    if (e != cudaSuccess)
        return cuda_fail(e);
    return 0;
}

} // namespace

extern "C" {

int posit_init(void)
{
    int r = ensure_init();
    if (r)
        return r;
    PG_TRY(cudaFree(nullptr)); // create the context
    return 0;
}

size_t posit_rgemm_workspace_size(char transa, char transb, int m, int n, int k)
{
    (void)transa;
    (void)transb;
    if (m <= 0 || n <= 0 || k <= 0)
        return 0;
    return pg::gemm_workspace_bytes(m, n, k);
}

int posit_rgemm_dev(char transa, char transb, int m, int n, int k, uint32_t alpha, const uint32_t *A,
                    int lda, const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc, void *workspace,
                    size_t workspace_bytes, void *stream)
{
    bool nota, notb;
    int info = rgemm_check_args(transa, transb, m, n, k, lda, ldb, ldc, nota, notb);
    if (info)
        return info;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamPerThread;
    return rgemm_device(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace, workspace_bytes, st);
}

int posit_rgemm(char transa, char transb, int m, int n, int k, uint32_t alpha, const uint32_t *A, int lda,
                const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc)
{
    bool nota, notb;
    int info = rgemm_check_args(transa, transb, m, n, k, lda, ldb, ldc, nota, notb);
    if (info)
        return info;
    if (m == 0 || n == 0 || ((alpha == 0 || k == 0) && beta == pg::P32_ONE))
        return 0;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = cudaStreamPerThread;
    const bool need_ab = !(alpha == 0 || k == 0);
    // device copies of exactly the referenced submatrices, packed (ld = rows)
    const int ar = nota ? m : k, ac = nota ? k : m;
    const int br = notb ? k : n, bc = notb ? n : k;
    uint32_t *dA = nullptr, *dB = nullptr, *dC = nullptr;
    PG_TRY(cudaMallocAsync((void **)&dC, (size_t)m * n * 4, st));
    if (need_ab) {
        PG_TRY(cudaMallocAsync((void **)&dA, (size_t)ar * ac * 4, st));
        PG_TRY(cudaMallocAsync((void **)&dB, (size_t)br * bc * 4, st));
        PG_TRY(cudaMemcpy2DAsync(dA, (size_t)ar * 4, A, (size_t)lda * 4, (size_t)ar * 4, ac,
                                 cudaMemcpyHostToDevice, st));
        PG_TRY(cudaMemcpy2DAsync(dB, (size_t)br * 4, B, (size_t)ldb * 4, (size_t)br * 4, bc,
                                 cudaMemcpyHostToDevice, st));
    }
    if (beta != 0) // with beta == 0 the reference never reads C (Rgemm.cpp:143-147, 170-173, 197-198)
        PG_TRY(cudaMemcpy2DAsync(dC, (size_t)m * 4, C, (size_t)ldc * 4, (size_t)m * 4, n,
                                 cudaMemcpyHostToDevice, st));
    int rc = rgemm_device(nota, notb, m, n, k, alpha, dA, ar, dB, br, beta, dC, m, nullptr, 0, st);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy2DAsync(C, (size_t)ldc * 4, dC, (size_t)m * 4, (size_t)m * 4, n,
                                          cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            rc = cuda_fail(e);
    }
    if (dA)
        cudaFreeAsync(dA, st);
    if (dB)
        cudaFreeAsync(dB, st);
    cudaFreeAsync(dC, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == 0 && e != cudaSuccess)
        rc = cuda_fail(e);
    if (rc == 0 && pg::read_device_error(true) != 0)
        rc = POSIT_E_DEVICE_FAULT;
    return rc;
}

// ---- factorizations -------------------------------------------------------------
static int pick_nb(int nb, bool lu, int n) { return nb > 0 ? nb : pg::tuned_panel_width(lu, n); }
static cudaStream_t as_stream(void *stream) { return stream ? (cudaStream_t)stream : cudaStreamPerThread; }

int posit_rgetrf_dev(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info, void *stream)
{
    if (m < 0)
        return 1; // Rgetrf.cpp:60-66
    if (n < 0)
        return 2;
    if (lda < imax(1, m))
        return 4;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = as_stream(stream);
    PG_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
    if (m == 0 || n == 0)
        return 0;
    nb = pick_nb(nb, true, m < n ? m : n);
    void *ws = nullptr;
    PG_TRY(cudaMallocAsync(&ws, pg::rgetrf_workspace_bytes(m, n, nb), st));
    cudaError_t e = pg::rgetrf_launch(m, n, A, lda, ipiv, nb, info, ws, st);
    cudaFreeAsync(ws, st);
    return e == cudaSuccess ? 0 : cuda_fail(e);
}

int posit_rgetrs_dev(char trans, int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B,
                     int ldb, void *stream)
{
    bool notr = same(trans, 'N');
    if (!notr && !same(trans, 'T') && !same(trans, 'C'))
        return 1; // Rgetrs.cpp:60-71
    if (n < 0)
        return 2;
    if (nrhs < 0)
        return 3;
    if (lda < imax(1, n))
        return 5;
    if (ldb < imax(1, n))
        return 8;
    int r = ensure_init();
    if (r)
        return r;
    if (n == 0 || nrhs == 0)
        return 0;
    if (notr)
        PG_TRY(pg::rgetrs_launch(n, nrhs, A, lda, ipiv, B, ldb, as_stream(stream)));
    else
        PG_TRY(pg::rgetrs_trans_launch(n, nrhs, A, lda, ipiv, B, ldb, as_stream(stream)));
    return 0;
}

int posit_tuned_panel_width(int lu, int n) { return pg::tuned_panel_width(lu != 0, n); }

int posit_rpotrf_dev(char uplo, int n, uint32_t *A, int lda, int nb, int *info, void *stream)
{
    bool upper = same(uplo, 'U');
    if (!upper && !same(uplo, 'L'))
        return 1; // Rpotrf.cpp:64-72
    if (n < 0)
        return 2;
    if (lda < imax(1, n))
        return 4;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = as_stream(stream);
    PG_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
    if (n == 0)
        return 0;
    // the upper factor depends on nb: the default is the reference's own block size
    nb = upper ? (nb > 0 ? nb : POSIT_RPOTRF_UPPER_DEFAULT_NB) : pick_nb(nb, false, n);
    const size_t wsb = upper ? pg::rpotrf_upper_workspace_bytes(n, nb) : pg::rpotrf_workspace_bytes(n, nb);
    void *ws = nullptr;
    if (wsb)
        PG_TRY(cudaMallocAsync(&ws, wsb, st));
    cudaError_t e = upper ? pg::rpotrf_upper_launch(n, A, lda, nb, info, ws, st)
                          : pg::rpotrf_lower_launch(n, A, lda, nb, info, ws, st);
    if (ws)
        cudaFreeAsync(ws, st);
    return e == cudaSuccess ? 0 : cuda_fail(e);
}

int posit_rpotrs_dev(char uplo, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb, void *stream)
{
    bool upper = same(uplo, 'U');
    if (!upper && !same(uplo, 'L'))
        return 1; // Rpotrs.cpp:60-71
    if (n < 0)
        return 2;
    if (nrhs < 0)
        return 3;
    if (lda < imax(1, n))
        return 5;
    if (ldb < imax(1, n))
        return 7;
    int r = ensure_init();
    if (r)
        return r;
    if (n == 0 || nrhs == 0)
        return 0;
    if (upper)
        PG_TRY(pg::rpotrs_upper_launch(n, nrhs, A, lda, B, ldb, as_stream(stream)));
    else
        PG_TRY(pg::rpotrs_lower_launch(n, nrhs, A, lda, B, ldb, as_stream(stream)));
    return 0;
}

// Host forms: copy the referenced parts to the device, run, copy back, synchronise.
static int finish(cudaStream_t st, int rc)
{
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == 0 && e != cudaSuccess)
        rc = cuda_fail(e);
    if (rc == 0 && pg::read_device_error(true) != 0)
        rc = POSIT_E_DEVICE_FAULT;
    return rc;
}

int posit_rgetrf(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info)
{
    if (m < 0)
        return 1;
    if (n < 0)
        return 2;
    if (lda < imax(1, m))
        return 4;
    *info = 0;
    if (m == 0 || n == 0)
        return 0;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = cudaStreamPerThread;
    uint32_t *dA = nullptr;
    int *dp = nullptr;
    const int mn = m < n ? m : n;
    PG_TRY(cudaMallocAsync((void **)&dA, (size_t)m * n * 4, st));
    PG_TRY(cudaMallocAsync((void **)&dp, ((size_t)mn + 1) * sizeof(int), st));
    PG_TRY(cudaMemcpy2DAsync(dA, (size_t)m * 4, A, (size_t)lda * 4, (size_t)m * 4, n, cudaMemcpyHostToDevice, st));
    int rc = posit_rgetrf_dev(m, n, dA, m, dp + 1, nb, dp, st);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy2DAsync(A, (size_t)lda * 4, dA, (size_t)m * 4, (size_t)m * 4, n,
                                          cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ipiv, dp + 1, (size_t)mn * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(info, dp, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            rc = cuda_fail(e);
    }
    cudaFreeAsync(dA, st);
    cudaFreeAsync(dp, st);
    return finish(st, rc);
}

int posit_rgetrs(char trans, int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb)
{
    bool notr = same(trans, 'N');
    if (!notr && !same(trans, 'T') && !same(trans, 'C'))
        return 1;
    if (n < 0)
        return 2;
    if (nrhs < 0)
        return 3;
    if (lda < imax(1, n))
        return 5;
    if (ldb < imax(1, n))
        return 8;
    if (n == 0 || nrhs == 0)
        return 0;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = cudaStreamPerThread;
    uint32_t *dA = nullptr, *dB = nullptr;
    int *dp = nullptr;
    PG_TRY(cudaMallocAsync((void **)&dA, (size_t)n * n * 4, st));
    PG_TRY(cudaMallocAsync((void **)&dB, (size_t)n * nrhs * 4, st));
    PG_TRY(cudaMallocAsync((void **)&dp, (size_t)n * sizeof(int), st));
    PG_TRY(cudaMemcpy2DAsync(dA, (size_t)n * 4, A, (size_t)lda * 4, (size_t)n * 4, n, cudaMemcpyHostToDevice, st));
    PG_TRY(cudaMemcpy2DAsync(dB, (size_t)n * 4, B, (size_t)ldb * 4, (size_t)n * 4, nrhs, cudaMemcpyHostToDevice, st));
    PG_TRY(cudaMemcpyAsync(dp, ipiv, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
    int rc = posit_rgetrs_dev(trans, n, nrhs, dA, n, dp, dB, n, st);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy2DAsync(B, (size_t)ldb * 4, dB, (size_t)n * 4, (size_t)n * 4, nrhs,
                                          cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            rc = cuda_fail(e);
    }
    cudaFreeAsync(dA, st);
    cudaFreeAsync(dB, st);
    cudaFreeAsync(dp, st);
    return finish(st, rc);
}

int posit_rpotrf(char uplo, int n, uint32_t *A, int lda, int nb, int *info)
{
    bool upper = same(uplo, 'U');
    if (!upper && !same(uplo, 'L'))
        return 1;
    if (n < 0)
        return 2;
    if (lda < imax(1, n))
        return 4;
    *info = 0;
    if (n == 0)
        return 0;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = cudaStreamPerThread;
    uint32_t *dA = nullptr;
    int *di = nullptr;
    PG_TRY(cudaMallocAsync((void **)&dA, (size_t)n * n * 4, st));
    PG_TRY(cudaMallocAsync((void **)&di, sizeof(int), st));
    PG_TRY(cudaMemcpy2DAsync(dA, (size_t)n * 4, A, (size_t)lda * 4, (size_t)n * 4, n, cudaMemcpyHostToDevice, st));
    int rc = posit_rpotrf_dev(uplo, n, dA, n, nb, di, st);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy2DAsync(A, (size_t)lda * 4, dA, (size_t)n * 4, (size_t)n * 4, n,
                                          cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(info, di, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            rc = cuda_fail(e);
    }
    cudaFreeAsync(dA, st);
    cudaFreeAsync(di, st);
    return finish(st, rc);
}

int posit_rpotrs(char uplo, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb)
{
    bool upper = same(uplo, 'U');
    if (!upper && !same(uplo, 'L'))
        return 1;
    if (n < 0)
        return 2;
    if (nrhs < 0)
        return 3;
    if (lda < imax(1, n))
        return 5;
    if (ldb < imax(1, n))
        return 7;
    if (n == 0 || nrhs == 0)
        return 0;
    int r = ensure_init();
    if (r)
        return r;
    cudaStream_t st = cudaStreamPerThread;
    uint32_t *dA = nullptr, *dB = nullptr;
    PG_TRY(cudaMallocAsync((void **)&dA, (size_t)n * n * 4, st));
    PG_TRY(cudaMallocAsync((void **)&dB, (size_t)n * nrhs * 4, st));
    PG_TRY(cudaMemcpy2DAsync(dA, (size_t)n * 4, A, (size_t)lda * 4, (size_t)n * 4, n, cudaMemcpyHostToDevice, st));
    PG_TRY(cudaMemcpy2DAsync(dB, (size_t)n * 4, B, (size_t)ldb * 4, (size_t)n * 4, nrhs, cudaMemcpyHostToDevice, st));
    int rc = posit_rpotrs_dev(uplo, n, nrhs, dA, n, dB, n, st);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy2DAsync(B, (size_t)ldb * 4, dB, (size_t)n * 4, (size_t)n * 4, nrhs,
                                          cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            rc = cuda_fail(e);
    }
    cudaFreeAsync(dA, st);
    cudaFreeAsync(dB, st);
    return finish(st, rc);
}

int posit_from_double_dev(const double *x, uint32_t *out, size_t n, void *stream)
{
    int r = ensure_init();
    if (r)
        return r;
    PG_TRY(pg::convert_launch(true, x, out, n, stream ? (cudaStream_t)stream : cudaStreamPerThread));
    return 0;
}

int posit_to_double_dev(const uint32_t *x, double *out, size_t n, void *stream)
{
    int r = ensure_init();
    if (r)
        return r;
    PG_TRY(pg::convert_launch(false, x, out, n, stream ? (cudaStream_t)stream : cudaStreamPerThread));
    return 0;
}

int posit_device_error(int clear) { return pg::read_device_error(clear != 0); }

void posit_profile_enable(int on) { pg::profile_enable(on != 0); }

int posit_profile_read(double *main_kernel_ms, long long *main_launches, long long *all_launches, int reset)
{
    return pg::profile_read(main_kernel_ms, main_launches, all_launches, reset != 0);
}

int posit_last_cuda_error(void) { return g_last_cuda_error.load(); }

const char *posit_strerror(int code)
{
    switch (code) {
    case 0:
        return "success";
    case POSIT_E_CUDA:
        return "CUDA runtime error";
    case POSIT_E_NO_DEVICE:
        return "no usable CUDA device";
    case POSIT_E_NO_MEMORY:
        return "out of device memory";
    case POSIT_E_DEVICE_FAULT:
        return "kernel error flag raised (bounded wait expired)";
    case POSIT_E_WORKSPACE:
        return "workspace too small or misaligned";
    case POSIT_E_UNSUPPORTED:
        return "variant not implemented on the device";
    case POSIT_E_NOALLOC_LIMIT:
        return "shape needs more scratch than the allocation-free entry point's static array";
    case POSIT_E_QUEUE_FULL:
        return "server queue full";
    case POSIT_E_CANCELLED:
        return "request cancelled";
    case POSIT_E_NOT_CACHED:
        return "no factor cached under this matrix id";
    case POSIT_E_MISMATCH:
        return "matrix id cached with another kind or order";
    case POSIT_E_UNKNOWN_TICKET:
        return "unknown ticket";
    default:
        if (code > 0)
            return "illegal argument (BLAS info = parameter number)";
        return "unknown error";
    }
}

} // extern "C"
