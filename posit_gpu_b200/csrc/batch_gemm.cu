// batch_gemm.cu -- many independent posit32 GEMMs of uneven shapes in one persistent
// launch fed by a device work queue of output tiles.
//
// The queue holds (problem, tile row, tile column, tile shape) items sorted by
// decreasing k.  A CTA takes the next item, loads its operands straight from the
// problem's matrices into FP64 tiles (transposes and alpha*B for the NN/NT order handled
// during the load), and runs the same k-step routine as the single-GEMM kernel
// (gemm_tile.cuh, tile_steps_f64), so
// every C is bit-identical to posit_rgemm_dev's, i.e. to the CPU Rgemm.  Three tile
// shapes (64x32, 32x32, 32x64 outputs per CTA) cover small and skinny problems; which one
// a problem uses comes from a table indexed by its (m, n) size bucket, produced by the
// autotuner (posit_gpu_b200/autotune.py).
#include "batch_gemm.cuh"
#include "gemm.cuh"
#include "gemm_tile.cuh"
#include "posit32.cuh"

namespace pg {

namespace {

constexpr int BG_THREADS = 256;
constexpr int BG_MAXB = 64; // largest tile side

template <int TM_, int TN_>
__device__ void batch_tile(const BatchGemmDesc &P, int mt, int nt, double *As, double *Ts, unsigned char *rnar,
                           unsigned char *cnar, const double *ctab)
{
    constexpr int BM_ = 16 * TM_, BN_ = 16 * TN_;
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const bool nota = P.nota != 0, notb = P.notb != 0, dot = !nota;
    const int m = P.m, n = P.n, k = P.k;
    for (int i = tid; i < BM_; i += BG_THREADS)
        rnar[i] = 0;
    for (int j = tid; j < BN_; j += BG_THREADS)
        cnar[j] = 0;
    double acc[TM_][TN_];
    uint32_t nar_bits = 0;
#pragma unroll
    for (int i = 0; i < TM_; ++i) {
#pragma unroll
        for (int j = 0; j < TN_; ++j) {
            const int row = mt * BM_ + own_off(tx, i), col = nt * BN_ + own_off(ty, j);
            uint32_t u = 0;
            if (!dot) {
                u = P32_ONE;
                if (row < m && col < n) {
                    u = P.C[(size_t)row + (size_t)col * P.ldc];
                    if (P.beta == 0)
                        u = 0;
                    else if (P.beta != P32_ONE)
                        u = pmul(P.beta, u);
                }
                if (u == P32_NAR) {
                    nar_bits |= 1u << (i * TN_ + j);
                    u = P32_ONE;
                }
            }
            acc[i][j] = p32_to_double(u);
        }
    }
    __syncthreads();
    const int KT = (k + BK - 1) / BK;
    for (int kt = 0; kt < KT; ++kt) {
        for (int e = tid; e < BM_ * BK; e += BG_THREADS) {
            const int i = e % BM_, l = e / BM_;
            const int row = mt * BM_ + i, kk = kt * BK + l;
            uint32_t u = P32_ONE;
            if (row < m && kk < k)
                u = nota ? P.A[(size_t)row + (size_t)kk * P.lda] : P.A[(size_t)kk + (size_t)row * P.lda];
            if (u == P32_NAR) {
                rnar[i] = 1;
                u = P32_ONE;
            }
            As[l * BM_ + i] = p32_to_double(u);
        }
        for (int e = tid; e < BK * BN_; e += BG_THREADS) {
            const int j = e % BN_, l = e / BN_;
            const int col = nt * BN_ + j, kk = kt * BK + l;
            uint32_t u = P32_ONE;
            if (col < n && kk < k) {
                u = notb ? P.B[(size_t)kk + (size_t)col * P.ldb] : P.B[(size_t)col + (size_t)kk * P.ldb];
                if (!dot)
                    u = pmul(P.alpha, u); // Rgemm.cpp:180 / 222
            }
            if (u == P32_NAR) {
                cnar[j] = 1;
                u = P32_ONE;
            }
            Ts[l * BN_ + j] = p32_to_double(u);
        }
        __syncthreads();
        tile_steps_f64<TM_, TN_>(acc, As, Ts, min(BK, k - kt * BK), ctab, tx, ty);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM_; ++i) {
#pragma unroll
        for (int j = 0; j < TN_; ++j) {
            const int li = own_off(tx, i), lj = own_off(ty, j);
            const int row = mt * BM_ + li, col = nt * BN_ + lj;
            if (row < m && col < n) {
                uint32_t *cp = P.C + (size_t)row + (size_t)col * P.ldc;
                const bool nar = ((nar_bits >> (i * TN_ + j)) & 1u) || rnar[li] || cnar[lj];
                uint32_t v = nar ? P32_NAR : p32_from_double(acc[i][j]);
                if (dot) {
                    uint32_t at = pmul(P.alpha, v);
                    v = (P.beta == 0) ? at : padd(at, pmul(P.beta, *cp));
                }
                *cp = v;
            }
        }
    }
}

// alpha == 0 or k == 0 with beta != 1, on the tile: C <- 0 or beta*C (alpha == 0,
// Rgemm.cpp:142-156; NN/NT with k == 0, Rgemm.cpp:169-177).  TN/TT with k == 0 and
// alpha != 0 form alpha*0 and combine it with beta*C (Rgemm.cpp:193-201): NaR when alpha
// is NaR.
__device__ void batch_scale_tile(const BatchGemmDesc &P, int mt, int nt, int bm, int bn)
{
    const bool dot = P.alpha != 0 && !P.nota;
    const uint32_t t = pmul(P.alpha, 0u);
    for (int e = threadIdx.x; e < bm * bn; e += BG_THREADS) {
        const int row = mt * bm + e % bm, col = nt * bn + e / bm;
        if (row < P.m && col < P.n) {
            uint32_t *cp = P.C + (size_t)row + (size_t)col * P.ldc;
            if (dot)
                *cp = (P.beta == 0) ? t : padd(t, pmul(P.beta, *cp));
            else
                *cp = (P.beta == 0) ? 0u : pmul(P.beta, *cp);
        }
    }
}

} // namespace

__global__ void __launch_bounds__(BG_THREADS, 2)
    batch_gemm_kernel(const BatchGemmDesc *__restrict__ probs, const BatchTile *__restrict__ tiles, int ntiles,
                      int *__restrict__ next)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double *ctab = reinterpret_cast<double *>(smem); // rounding constants (F64ConstTable8)
    double *As = reinterpret_cast<double *>(smem + (size_t)F64_CONST_ENTRIES * sizeof(double));
    double *Ts = As + BK * BG_MAXB;
    unsigned char *rnar = reinterpret_cast<unsigned char *>(Ts + BK * BG_MAXB);
    unsigned char *cnar = rnar + BG_MAXB;
    __shared__ int s_item;
    for (int i = threadIdx.x; i < F64_CONST_ENTRIES; i += BG_THREADS)
        ctab[i] = f64_from_hi(f64_round_const_top(i));
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(next, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= ntiles)
            return;
        const BatchTile t = tiles[item];
        const BatchGemmDesc P = probs[t.prob];
        const int bm = batch_tile_rows(t.cfg), bn = batch_tile_cols(t.cfg);
        if (P.alpha == 0 || P.k == 0)
            batch_scale_tile(P, t.mt, t.nt, bm, bn);
        else if (t.cfg == 0)
            batch_tile<4, 2>(P, t.mt, t.nt, As, Ts, rnar, cnar, ctab);
        else if (t.cfg == 1)
            batch_tile<2, 2>(P, t.mt, t.nt, As, Ts, rnar, cnar, ctab);
        else
            batch_tile<2, 4>(P, t.mt, t.nt, As, Ts, rnar, cnar, ctab);
        __syncthreads();
    }
}

size_t batch_gemm_smem_bytes()
{
    return (size_t)F64_CONST_ENTRIES * sizeof(double) + 2 * (size_t)BK * BG_MAXB * sizeof(double) + 2 * BG_MAXB;
}

cudaError_t batch_gemm_launch(const BatchGemmDesc *probs, const BatchTile *tiles, int ntiles, int *next, int ctas,
                              cudaStream_t st)
{
    const size_t smem = batch_gemm_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(batch_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    e = cudaMemsetAsync(next, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return e;
    batch_gemm_kernel<<<ctas, BG_THREADS, smem, st>>>(probs, tiles, ntiles, next);
    return cudaGetLastError();
}

} // namespace pg
