// gemm.cu -- bit-exact posit32 GEMM for sm_100a.
//
// Reproduces the per-element operation order of the reference CPU Rgemm
// (libRpack/Rgemm.cpp:163-247):
//   NN / NT  "scale, then accumulate":  c <- beta*c (0 if beta == 0, untouched if
//            beta == 1), then c <- c + (alpha*b_lj)*a_il for l = 0..k-1;
//   TN / TT  "dot, then combine":       t <- 0, t <- t + a_li*b_lj for l = 0..k-1,
//            then c <- alpha*t (beta == 0) or alpha*t + beta*c.
// Both are one chain of "acc <- acc + x_l*y_l" per output; they differ only in the
// operand prescale (alpha*B for NN/NT), the accumulator's start value and the
// epilogue.  So one main kernel serves all four transpose cases:
//
//  1. decode pre-pass: op(A) and op(B) (times alpha for NN/NT, rounded exactly as the
//     reference rounds alpha*b_lj) are converted ONCE per element to FP64 (posit32
//     values are exact there), stored tile-contiguously in a workspace: A as
//     [m-tile][k-tile][l][i], B as [n-tile][k-tile][l][j], plus a NaR flag per row and
//     column.  Transposition is absorbed here, so the main kernel never sees lda/ldb.
//  2. main kernel: one CTA per 64x32 tile of C, 256 threads, 4x2 outputs per thread held
//     in FP64 across the whole k loop (two sets taking turns, gemm_tile.cuh), 3 CTAs per
//     SM.  Each 16-deep k tile of A and B
//     (8 KB + 4 KB) is brought into shared memory by the bulk-copy (TMA) engine
//     (cp.async.bulk + mbarrier transaction counts, 3 stages, every wait bounded).  The
//     inner step is the FP64 form of p32_mul + p32_add (posit32.cuh, f64_posit_mac) with
//     the rounding constants in a shared-memory table, written into the other accumulator
//     set without a select; the rare step it flags (an inexact FP64 sum, a result outside
//     the fast window) is redone exactly from the set it read, in order, right after its
//     k step.
#include "gemm.cuh"
#include "gemm_tile.cuh"
#include "posit32.cuh"

#include <atomic>
#include <mutex>
#include <vector>

namespace pg {

__device__ int g_dev_error;

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier + bulk async copy (TMA engine, no multicast)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

// Every wait is bounded: a copy that never lands turns into an error flag, not a hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t it = 0; it < (1u << 24); ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

GemmPlan gemm_plan(int m, int n, int k)
{
    GemmPlan p;
    p.m = m;
    p.n = n;
    p.k = k;
    p.mt = (m + BM - 1) / BM;
    p.nt = (n + BN - 1) / BN;
    p.kt = (k + BK - 1) / BK;
    p.a_bytes = (size_t)p.mt * p.kt * BK * BM * sizeof(double);
    p.b_bytes = (size_t)p.nt * p.kt * BK * BN * sizeof(double);
    p.flag_bytes = (size_t)(p.mt * BM + p.nt * BN);
    return p;
}

size_t gemm_workspace_bytes(int m, int n, int k)
{
    GemmPlan p = gemm_plan(m, n, k);
    return p.a_bytes + p.b_bytes + p.flag_bytes;
}

// ---------------------------------------------------------------------------
// Decode pre-pass
// ---------------------------------------------------------------------------
// op(A) (m x k) -> Ad[mt][kt][l][i].  Rows/columns beyond the matrix hold 1.0 so that
// padded lanes stay on the fast path; their results are never stored.
// A NaR operand makes every output of its row NaR (p32_mul and p32_add propagate NaR,
// kernel_entry.cl:385-390, 414-417); that is recorded in row_nar[] and the operand is
// decoded as 1.0 so the row's arithmetic stays on the fast path.
__global__ void decode_a_kernel(bool nota, int m, int k, const uint32_t *__restrict__ A, size_t lda,
                                int KT, size_t total, double *__restrict__ Ad, unsigned char *__restrict__ row_nar)
{
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(idx % BM);
        size_t r = idx / BM;
        int l = (int)(r % BK);
        r /= BK;
        int kt = (int)(r % KT);
        int mt = (int)(r / KT);
        int row = mt * BM + i, kk = kt * BK + l;
        uint32_t u = P32_ONE;
        if (row < m && kk < k)
            u = nota ? A[(size_t)row + (size_t)kk * lda] : A[(size_t)kk + (size_t)row * lda];
        if (u == P32_NAR) {
            row_nar[row] = 1;
            u = P32_ONE;
        }
        Ad[idx] = p32_to_double(u);
    }
}

// op(B) (k x n) -> Td[nt][kt][l][j], times alpha (exactly rounded) when `scale`.
__global__ void decode_b_kernel(bool notb, int k, int n, const uint32_t *__restrict__ B, size_t ldb,
                                bool scale, uint32_t alpha, int KT, size_t total, double *__restrict__ Td,
                                unsigned char *__restrict__ col_nar)
{
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(idx % BN);
        size_t r = idx / BN;
        int l = (int)(r % BK);
        r /= BK;
        int kt = (int)(r % KT);
        int nt = (int)(r / KT);
        int col = nt * BN + j, kk = kt * BK + l;
        uint32_t u = P32_ONE;
        if (col < n && kk < k) {
            u = notb ? B[(size_t)kk + (size_t)col * ldb] : B[(size_t)col + (size_t)kk * ldb];
            if (scale)
                u = pmul(alpha, u); // Rgemm.cpp:180 / 222: temp = alpha*b
        }
        if (u == P32_NAR) {
            col_nar[col] = 1;
            u = P32_ONE;
        }
        Td[idx] = p32_to_double(u);
    }
}

// ---------------------------------------------------------------------------
// Main kernel
// ---------------------------------------------------------------------------
// TRI selects the entries written: TRI_FULL all of C; TRI_LOWER only row >= column (the
// symmetric trailing update of a lower Cholesky factorization); TRI_UPPER only row <=
// column (Rsyrk('U', 'T') of an upper one).  Tiles wholly outside the triangle exit at once.
// `stop`, if given, is a device flag (a factorization's info) that turns the call into a
// no-op when it is nonzero.
template <bool DOT, int TRI>
__global__ void __launch_bounds__(NTHREADS, MIN_CTAS_PER_SM)
    gemm_main_kernel(int m, int n, int k, int KT, uint32_t alpha, uint32_t beta,
                     const double *__restrict__ Ad, const double *__restrict__ Td, uint32_t *__restrict__ C,
                     size_t ldc, const unsigned char *__restrict__ row_nar,
                     const unsigned char *__restrict__ col_nar, const int *__restrict__ stop)
{
    if (stop && *stop != 0)
        return;
    if (TRI == TRI_LOWER && (int)(blockIdx.x * BM + BM - 1) < (int)(blockIdx.y * BN))
        return; // every row of the tile is above its first column
    if (TRI == TRI_UPPER && (int)(blockIdx.x * BM) > (int)(blockIdx.y * BN + BN - 1))
        return; // every row of the tile is below its last column
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *As = reinterpret_cast<double *>(smem_raw);
    double *Ts = As + STAGES * BK * BM;
    double *ctab = Ts + STAGES * BK * BN; // rounding constants (F64ConstTable8)
    __shared__ __align__(8) uint64_t full[STAGES];

    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int mt = blockIdx.x, nt = blockIdx.y;
    const double *Ablk = Ad + (size_t)mt * KT * BK * BM;
    const double *Tblk = Td + (size_t)nt * KT * BK * BN;
    constexpr uint32_t kATileBytes = BK * BM * sizeof(double);
    constexpr uint32_t kBTileBytes = BK * BN * sizeof(double);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s)
            mbar_init(&full[s], 1);
        mbar_fence_init();
    }
    for (int i = tid; i < F64_CONST_ENTRIES; i += NTHREADS)
        ctab[i] = f64_from_hi(f64_round_const_top(i));
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < STAGES && s < KT; ++s) {
            mbar_arrive_expect_tx(&full[s], kATileBytes + kBTileBytes);
            bulk_g2s(As + s * BK * BM, Ablk + (size_t)s * BK * BM, kATileBytes, &full[s]);
            bulk_g2s(Ts + s * BK * BN, Tblk + (size_t)s * BK * BN, kBTileBytes, &full[s]);
        }
    }

    // Accumulators: NN/NT start from beta*C, TN/TT from zero.  A NaR start value is
    // remembered in nar_bits (the output stays NaR whatever follows) and replaced by 1.0.
    double acc[TM][TN];
    uint32_t nar_bits = 0;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int row = mt * BM + own_off(tx, i), col = nt * BN + own_off(ty, j);
            uint32_t u = 0;
            if (!DOT) {
                u = P32_ONE;
                if (row < m && col < n) {
                    u = C[(size_t)row + (size_t)col * ldc];
                    if (beta == 0)
                        u = 0; // Rgemm.cpp:170-173: C is not read
                    else if (beta != P32_ONE)
                        u = pmul(beta, u);
                }
                if (u == P32_NAR) {
                    nar_bits |= 1u << (i * TN + j);
                    u = P32_ONE;
                }
            }
            acc[i][j] = p32_to_double(u);
        }
    }

    bool bad = false;
    int kt_stop = 0;
    for (int kt = 0; kt < KT; ++kt) {
        kt_stop = kt;
        const int s = kt % STAGES;
        const uint32_t parity = (uint32_t)(kt / STAGES) & 1u;
        const bool arrived = mbar_wait_bounded(&full[s], parity);
        const double *as = As + s * BK * BM;
        const double *ts = Ts + s * BK * BN;
        const int lmax = min(BK, k - kt * BK);
        tile_steps_f64<TM, TN>(acc, as, ts, lmax, ctab, tx, ty);
        // every thread is done with stage s before it is refilled
        bad = __syncthreads_or(!arrived) != 0;
        if (bad)
            break;
        if (tid == 0 && kt + STAGES < KT) {
            const int nk = kt + STAGES;
            mbar_arrive_expect_tx(&full[s], kATileBytes + kBTileBytes);
            bulk_g2s(As + s * BK * BM, Ablk + (size_t)nk * BK * BM, kATileBytes, &full[s]);
            bulk_g2s(Ts + s * BK * BN, Tblk + (size_t)nk * BK * BN, kBTileBytes, &full[s]);
        }
    }

    if (bad) {
        if (tid == 0) {
            atomicOr(&g_dev_error, DEV_ERR_WAIT_TIMEOUT);
            // let copies already in flight land before the CTA's shared memory goes away
            for (int q = kt_stop + 1; q < KT && q < kt_stop + STAGES; ++q)
                (void)mbar_wait_bounded(&full[q % STAGES], (uint32_t)(q / STAGES) & 1u);
        }
        return;
    }

#pragma unroll
    for (int i = 0; i < TM; ++i) {
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int row = mt * BM + own_off(tx, i), col = nt * BN + own_off(ty, j);
            if (row < m && col < n && (TRI != TRI_LOWER || row >= col) && (TRI != TRI_UPPER || row <= col)) {
                uint32_t *cp = C + (size_t)row + (size_t)col * ldc;
                const bool nar = ((nar_bits >> (i * TN + j)) & 1u) || row_nar[row] || col_nar[col];
                uint32_t v = nar ? P32_NAR : p32_from_double(acc[i][j]);
                if (DOT) { // Rgemm.cpp:197-201
                    uint32_t at = pmul(alpha, v);
                    v = (beta == 0) ? at : padd(at, pmul(beta, *cp));
                }
                *cp = v;
            }
        }
    }
}

// C <- 0 or beta*C (alpha == 0, Rgemm.cpp:142-156; NN/NT with k == 0, Rgemm.cpp:169-177), or,
// with `dot`, the dot-then-combine epilogue of an empty sum (TN/TT with k == 0,
// Rgemm.cpp:193-201): t = alpha*0, then c = t (beta == 0) or t + beta*c.  alpha*0 is NaR
// when alpha is NaR (p32_mul tests NaR before zero, kernel_entry.cl:414-421).
__global__ void scale_kernel(int m, int n, bool dot, uint32_t alpha, uint32_t beta, uint32_t *__restrict__ C,
                             size_t ldc)
{
    size_t total = (size_t)m * n;
    const uint32_t t = pmul(alpha, 0u);
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        size_t i = idx % m, j = idx / m;
        uint32_t *cp = C + i + j * ldc;
        if (dot)
            *cp = (beta == 0) ? t : padd(t, pmul(beta, *cp));
        else
            *cp = (beta == 0) ? 0u : pmul(beta, *cp);
    }
}

// ---------------------------------------------------------------------------
// Instrumentation
// ---------------------------------------------------------------------------
namespace {
std::mutex g_prof_mu;
std::atomic<bool> g_prof_on{false};
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;
double g_prof_ms = 0.0;
long long g_prof_main = 0, g_prof_all = 0;

void prof_count(int launches)
{
    if (!g_prof_on)
        return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_all += launches;
}

cudaEvent_t prof_mark(cudaStream_t st)
{
    cudaEvent_t ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess)
        return nullptr;
    cudaEventRecord(ev, st);
    return ev;
}
} // namespace

void profile_enable(bool on)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = on;
}

int profile_read(double *main_ms, long long *main_launches, long long *all_launches, bool reset)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto &pr : g_prof_events) {
        float ms = 0.f;
        if (pr.first && pr.second && cudaEventSynchronize(pr.second) == cudaSuccess &&
            cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess)
            g_prof_ms += ms;
        if (pr.first)
            cudaEventDestroy(pr.first);
        if (pr.second)
            cudaEventDestroy(pr.second);
        g_prof_main += 1;
    }
    g_prof_events.clear();
    if (main_ms)
        *main_ms = g_prof_ms;
    if (main_launches)
        *main_launches = g_prof_main;
    if (all_launches)
        *all_launches = g_prof_all;
    if (reset) {
        g_prof_ms = 0.0;
        g_prof_main = 0;
        g_prof_all = 0;
    }
    return 0;
}

__global__ void from_double_kernel(const double *__restrict__ x, uint32_t *__restrict__ out, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = p32_from_double(x[i]);
}

__global__ void to_double_kernel(const uint32_t *__restrict__ x, double *__restrict__ out, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = p32_to_double(x[i]);
}

static int grid_for(size_t total, int threads)
{
    size_t b = (total + threads - 1) / threads;
    size_t cap = 148 * 16;
    return (int)(b < cap ? (b ? b : 1) : cap);
}

template <int TRI>
static cudaError_t gemm_launch_impl(bool nota, bool notb, int m, int n, int k, uint32_t alpha, const uint32_t *A,
                                    int lda, const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc,
                                    void *workspace, cudaStream_t stream, const int *stop)
{
    GemmPlan p = gemm_plan(m, n, k);
    double *Ad = reinterpret_cast<double *>(workspace);
    double *Td = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(workspace) + p.a_bytes);
    unsigned char *row_nar = reinterpret_cast<unsigned char *>(workspace) + p.a_bytes + p.b_bytes;
    unsigned char *col_nar = row_nar + (size_t)p.mt * BM;
    const bool dot = !nota; // TN / TT use the dot-then-combine order
    size_t na = p.a_bytes / sizeof(double), nb = p.b_bytes / sizeof(double);
    cudaError_t e = cudaMemsetAsync(row_nar, 0, p.flag_bytes, stream);
    if (e != cudaSuccess)
        return e;
    decode_a_kernel<<<grid_for(na, 256), 256, 0, stream>>>(nota, m, k, A, (size_t)lda, p.kt, na, Ad, row_nar);
    decode_b_kernel<<<grid_for(nb, 256), 256, 0, stream>>>(notb, k, n, B, (size_t)ldb, !dot, alpha, p.kt, nb,
                                                           Td, col_nar);
    const size_t smem = (size_t)STAGES * BK * (BM + BN) * sizeof(double) + (size_t)F64_CONST_ENTRIES * sizeof(double);
    dim3 grid(p.mt, p.nt);
    e = dot ? cudaFuncSetAttribute(gemm_main_kernel<true, TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem)
            : cudaFuncSetAttribute(gemm_main_kernel<false, TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem);
    if (e != cudaSuccess)
        return e;
    const bool prof = g_prof_on;
    cudaEvent_t e0 = prof ? prof_mark(stream) : nullptr;
    if (dot)
        gemm_main_kernel<true, TRI><<<grid, NTHREADS, smem, stream>>>(m, n, k, p.kt, alpha, beta, Ad, Td, C,
                                                                        (size_t)ldc, row_nar, col_nar, stop);
    else
        gemm_main_kernel<false, TRI><<<grid, NTHREADS, smem, stream>>>(m, n, k, p.kt, alpha, beta, Ad, Td, C,
                                                                         (size_t)ldc, row_nar, col_nar, stop);
    if (prof) {
        cudaEvent_t e1 = prof_mark(stream);
        std::lock_guard<std::mutex> lk(g_prof_mu);
        g_prof_events.emplace_back(e0, e1);
    }
    prof_count(3);
    return cudaGetLastError();
}

cudaError_t gemm_launch(bool nota, bool notb, int m, int n, int k, uint32_t alpha, const uint32_t *A, int lda,
                        const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc, void *workspace,
                        cudaStream_t stream)
{
    return gemm_launch_impl<TRI_FULL>(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace, stream,
                                      nullptr);
}

cudaError_t gemm_launch_tri(int tri, bool nota, bool notb, int m, int n, int k, uint32_t alpha, const uint32_t *A,
                            int lda, const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc,
                            void *workspace, cudaStream_t stream, const int *stop)
{
    if (tri == TRI_LOWER)
        return gemm_launch_impl<TRI_LOWER>(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace,
                                           stream, stop);
    if (tri == TRI_UPPER)
        return gemm_launch_impl<TRI_UPPER>(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace,
                                           stream, stop);
    return gemm_launch_impl<TRI_FULL>(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace, stream,
                                      stop);
}

cudaError_t gemm_launch_lower(bool nota, bool notb, int m, int n, int k, uint32_t alpha, const uint32_t *A, int lda,
                              const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc, void *workspace,
                              cudaStream_t stream, const int *stop)
{
    return gemm_launch_impl<TRI_LOWER>(nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, workspace,
                                       stream, stop);
}

cudaError_t scale_launch(int m, int n, bool dot, uint32_t alpha, uint32_t beta, uint32_t *C, int ldc,
                         cudaStream_t stream)
{
    scale_kernel<<<grid_for((size_t)m * n, 256), 256, 0, stream>>>(m, n, dot, alpha, beta, C, (size_t)ldc);
    prof_count(1);
    return cudaGetLastError();
}

cudaError_t convert_launch(bool to_posit, const void *in, void *out, size_t n, cudaStream_t stream)
{
    if (n == 0)
        return cudaSuccess;
    if (to_posit)
        from_double_kernel<<<grid_for(n, 256), 256, 0, stream>>>((const double *)in, (uint32_t *)out, n);
    else
        to_double_kernel<<<grid_for(n, 256), 256, 0, stream>>>((const uint32_t *)in, (double *)out, n);
    prof_count(1);
    return cudaGetLastError();
}

cudaError_t device_error_address(int **p) { return cudaGetSymbolAddress((void **)p, g_dev_error); }

int read_device_error(bool clear)
{
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_dev_error, sizeof(int)) != cudaSuccess)
        return -1;
    if (clear && v) {
        int z = 0;
        cudaMemcpyToSymbol(g_dev_error, &z, sizeof(int));
    }
    return v;
}

} // namespace pg
