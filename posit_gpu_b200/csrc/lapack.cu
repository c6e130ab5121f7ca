// lapack.cu -- device-resident posit32 LU (Rgetrf) and Cholesky (Rpotrf), and their
// solves (Rgetrs, Rpotrs), bit-exact against the reference's CPU routines.
//
// Operation order.  In the reference every entry of L and U receives its updates as
// a <- a + (-u)*l (Rgemm's c + (alpha*b)*a with alpha = -1, Rgemm.cpp:180-182; Rtrsm's
// b - b_k*a, Rtrsm.cpp:151, is the same bits because posit multiplication is symmetric in
// sign) in ascending k, however Rgetrf/Rgetrf2/Rpotrf/Rpotrf2 group the columns into
// blocks; L entries are then multiplied by the reciprocal of the pivot (Rgetrf2.cpp:121-122,
// Rscal) or of the Cholesky diagonal (Rtrsm.cpp:265-268), diagonals of a Cholesky factor
// take a square root (Rpotrf2.cpp:97).  So LU and lower Cholesky are independent of the
// block size bit for bit (the zero-multiplier skips of Rtrsm/Rsyrk add zero and change
// nothing unless a NaR is present), and the device code may block the work its own way:
//
//   panel (nb columns)   two kernels per column, ordered by the kernel boundary alone:
//                        the pivot (LU: iRamax and the row interchange) or diagonal
//                        (Cholesky: square root) step of one CTA, then the scaling of
//                        the column and the rank-1 update of the rest of the panel over
//                        all rows in parallel;
//   U block row          Rtrsm("L","L","N","U") as one CTA per column;
//   row interchanges     Rlaswp on the columns outside the panel;
//   trailing update      the posit32 GEMM of gemm.cu (NN for LU; NT restricted to the
//                        lower triangle for Cholesky).
// The matrix never leaves the device.  Upper Cholesky (dot-then-combine order, block size
// dependent) is not implemented on the device.
#include "gemm.cuh"
#include "lapack.cuh"

#include <algorithm>
#include <cooperative_groups.h>
#include "posit32.cuh"
#include "trsm_chain.cuh"

namespace pg {

// ---------------------------------------------------------------------------
// LU panel
// ---------------------------------------------------------------------------
// Two launches per panel column k, synchronised only by the kernel boundary:
//   lu_update_kernel  blocks over (rows > k) x (groups of PANEL_CG columns in (k, jb)):
//                     l_i = a_ik scaled as Rgetrf2 does, a_ic += (-u_kc)*l_i.  Column k is
//                     only read; the first column group writes l_i to a scratch column.
//   lu_pivot_kernel   one block: the scratch column into column k, then the pivot step of
//                     column k+1 -- iRamax over the updated column, the interchange of the
//                     pivot row across the panel, the scaling decision.
constexpr int PANEL_ROWS = 128; // rows per update block (one per thread)
constexpr int PANEL_CG = 4;     // panel columns per update block

// Pivot decision of one column, shared by the two kernels of a panel step.
struct PivotInfo {
    int row;       // panel-local row of the pivot
    uint32_t piv;  // pivot value (after the interchange it sits at row k)
    int mode;      // 0: zero pivot (no scaling), 1: multiply by reciprocal, 2: divide
    uint32_t recip;
};

// Workspace of the panel kernels: the pivot/diagonal record and a scratch column of m
// entries, then the trailing GEMM's workspace.
static size_t panel_ws_bytes(int m) { return 256 + (((size_t)m * 4 + 255) & ~(size_t)255); }

// Copies the scaled multipliers of column `copy_col` (rows copy_col+1 .. M-1) from the
// scratch column into place (copy_col < 0: none), then, when k < jb, the pivot step of
// column k: iRamax (iRamax.cpp:65-71) over panel-local rows [k, M) -- the first index of
// the strict maximum of abs() in posit order (signed integer order of the patterns, NaR
// lowest) -- the interchange of rows k and p over the panel's jb columns
// (Rgetrf2.cpp:107-117; with a zero pivot, over every column but k) and the scaling
// decision (Rgetrf2.cpp:119-131).
__global__ void __launch_bounds__(1024) lu_pivot_kernel(uint32_t *__restrict__ P, size_t lda, int M, int jb, int k,
                                                        int row0, int *__restrict__ ipiv, int *__restrict__ info,
                                                        PivotInfo *__restrict__ pinfo,
                                                        const uint32_t *__restrict__ lcol, int copy_col)
{
    __shared__ int32_t s_key[1024];
    __shared__ int s_idx[1024];
    if (*info < 0)
        return; // an earlier failure stops the factorization
    const int tid = threadIdx.x;
    if (copy_col >= 0) {
        uint32_t *pc = P + (size_t)copy_col * lda;
        for (int r = copy_col + 1 + tid; r < M; r += blockDim.x)
            pc[r] = lcol[r];
        __syncthreads(); // the interchange below moves two of these entries
    }
    if (k >= jb)
        return;
    int32_t best = INT32_MIN;
    int bidx = -1;
    const uint32_t *col = P + (size_t)k * lda;
    for (int i = k + tid; i < M; i += blockDim.x) {
        int32_t key = (int32_t)pabs(col[i]);
        if (bidx < 0 || key > best) { // rows visited in increasing order per thread
            best = key;
            bidx = i;
        }
    }
    // larger key wins, equal keys the smaller row; warp shuffles, then one warp over the
    // warps' results (blockDim.x == 1024: 32 warps)
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int round = 0; round < 2; ++round) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const int32_t k2 = __shfl_down_sync(0xFFFFFFFFu, best, off);
            const int i2 = __shfl_down_sync(0xFFFFFFFFu, bidx, off);
            if (i2 >= 0 && (bidx < 0 || k2 > best || (k2 == best && i2 < bidx))) {
                best = k2;
                bidx = i2;
            }
        }
        if (round == 0) {
            if (lane == 0) {
                s_key[warp] = best;
                s_idx[warp] = bidx;
            }
            __syncthreads();
            best = s_key[lane];
            bidx = s_idx[lane];
        }
    }
    if (tid == 0)
        s_idx[32] = bidx;
    __syncthreads();
    const int p = s_idx[32];
    const uint32_t piv = col[p];
    if (tid == 0) {
        ipiv[row0 + k] = row0 + p + 1; // 1-based, global
        PivotInfo pi;
        pi.row = p;
        pi.piv = piv;
        if (piv == 0) {
            pi.mode = 0;
            pi.recip = 0;
            if (*info == 0)
                *info = row0 + k + 1;
        } else if ((int32_t)pabs(piv) >= (int32_t)1u) { // |pivot| >= sfmin = FLT_MIN -> minpos
            pi.mode = 1;
            pi.recip = pdiv_est(P32_ONE, piv);
        } else {
            pi.mode = 2; // NaR pivot: element-wise division (Rgetrf2.cpp:124-126)
            pi.recip = 0;
        }
        *pinfo = pi;
    }
    __syncthreads(); // every thread has read the pivot before the rows move
    if (p != k) {
        // A zero pivot leaves its own column in place (Rgetrf2.cpp:107-117) while the
        // recursion's Rlaswp calls (Rgetrf2.cpp:141-150, 167-176) still move rows k and p in
        // every other column of the panel, and Rgetrf's outside it.
        for (int c = tid; c < jb; c += blockDim.x) {
            if (c == k && piv == 0)
                continue;
            uint32_t *pc = P + (size_t)c * lda;
            uint32_t t = pc[k];
            pc[k] = pc[p];
            pc[p] = t;
        }
    }
}

PG_HD uint32_t lu_scaled(uint32_t a, const PivotInfo &pi)
{
    if (pi.mode == 1)
        return pmul(pi.recip, a); // Rscal: da*dx
    if (pi.mode == 2)
        return pdiv_est(a, pi.piv);
    return a;
}

__global__ void __launch_bounds__(PANEL_ROWS) lu_update_kernel(uint32_t *__restrict__ P, size_t lda, int M, int jb,
                                                               int k, const int *__restrict__ info,
                                                               const PivotInfo *__restrict__ pinfo,
                                                               uint32_t *__restrict__ lcol)
{
    __shared__ double s_u[PANEL_CG]; // -u_kc for this block's columns, FP64
    if (*info < 0)
        return;
    const PivotInfo pi = *pinfo;
    const int c0 = k + 1 + blockIdx.y * PANEL_CG;
    if (threadIdx.x < PANEL_CG && c0 + (int)threadIdx.x < jb)
        s_u[threadIdx.x] = -p32_to_double(P[k + (size_t)(c0 + threadIdx.x) * lda]); // row k after the interchange
    __syncthreads();
    const int i = k + 1 + blockIdx.x * PANEL_ROWS + threadIdx.x;
    if (i >= M)
        return;
    const uint32_t l = lu_scaled(P[i + (size_t)k * lda], pi);
    if (blockIdx.y == 0)
        lcol[i] = l;
    const double dl = p32_to_double(l);
    const int cn = min(PANEL_CG, jb - c0);
    for (int j = 0; j < cn; ++j) { // a_ic + (-u_kc)*l_i in the FP64 step (posit32.cuh)
        uint32_t *pc = P + i + (size_t)(c0 + j) * lda;
        *pc = p32_from_double_exact(f64_posit_mac_checked(p32_to_double(*pc), s_u[j], dl));
    }
}

// ---------------------------------------------------------------------------
// LU panel in one thread-block cluster, held in shared memory: the per-column steps of
// lu_pivot_kernel + lu_update_kernel -- iRamax with first-max tie-break, the interchange
// across the panel, the scaling decision, the scaled column, the rank-1 update in the FP64
// step -- in the same per-element order, one launch per panel.  Up to 8 CTAs of T threads
// (T a multiple of 32, up to 1024).  The panel's rows are dealt out once, row i to CTA
// i mod ncta, and there to slot r of thread t with i / ncta = r*T + t (R slots per thread,
// jb FP64 values each, in shared memory); they never move: an interchange of rows k and p
// swaps the logical row numbers the two slots hold (each thread keeps its slots' numbers in
// registers, and every thread knows k and p, so each applies the swap to its own slots),
// and the write-back stores each slot at the row it holds at the end.  Per column, with the
// cluster's CTAs co-scheduled (no barrier waits for a CTA that never runs):
//   * each thread's best (key, logical row, value, slot) over its slots holding rows >= k,
//     reduced over the warp into the warp's slot in shared memory (double-buffered by
//     column parity); a cluster barrier (a block barrier with one CTA); every warp reduces
//     all warps' candidates, read through distributed shared memory -- every thread holds
//     the pivot, the same bits everywhere;
//   * threads read -u_kc from the pivot row's slot (in any CTA), one thread per CTA forms
//     the scaling decision and the reciprocal; a block barrier;
//   * each thread scales and updates its slots holding rows > k.
// The pivot row's slot is not written again in the panel (but for a zero pivot below row k,
// where the two slots trade back their column-k values: that column stays in place,
// Rgetrf2.cpp:107-117), so reading it after the candidates' barrier races with nothing.  A
// final cluster barrier keeps every CTA's shared memory alive until no other CTA reads it.
// ---------------------------------------------------------------------------
constexpr int PANEL1_THREADS = 1024;    // most threads per CTA
constexpr int PANEL1_MAX_JB = 512;
constexpr int PANEL1_MAX_CTAS = 8;
constexpr int PANEL1_SMEM_ENTRIES = 24; // R * jb * T <= 24 * 1024 FP64 values of shared memory per CTA
constexpr int PANEL1_MAX_R = 4;         // slots per thread (the LU panel keeps their row numbers in registers)
constexpr int PANEL1_ROWS_PER_CTA = 128; // the rows one CTA takes before another joins

// The barrier of a cluster panel: the cluster's, or the block's when the cluster is one CTA.
__device__ __forceinline__ void panel_sync(cooperative_groups::cluster_group &cl, int ncta)
{
    if (ncta == 1)
        __syncthreads();
    else
        cl.sync();
}

// Pivot key of an FP64-held posit value: |x|, NaR (NaN) below everything, the order of
// pabs() on patterns (iRamax.cpp:65-71 compares abs() in posit order).
__device__ __forceinline__ double pivot_key(double x) { return x != x ? -1.0 : fabs(x); }

// A pivot candidate: the largest key, the first (lowest logical row) among equal keys.
struct PivotCand {
    double key, val;
    int row;  // logical row, -1: none
    int slot; // (r << 16) | (CTA rank << 10) | thread of the slot holding it
};

__device__ __forceinline__ void cand_merge(PivotCand &a, const PivotCand &b)
{
    if (b.row >= 0 && (a.row < 0 || b.key > a.key || (b.key == a.key && b.row < a.row)))
        a = b;
}

__device__ __forceinline__ PivotCand cand_shfl_down(const PivotCand &a, int off)
{
    PivotCand b;
    b.key = __shfl_down_sync(0xFFFFFFFFu, a.key, off);
    b.val = __shfl_down_sync(0xFFFFFFFFu, a.val, off);
    b.row = __shfl_down_sync(0xFFFFFFFFu, a.row, off);
    b.slot = __shfl_down_sync(0xFFFFFFFFu, a.slot, off);
    return b;
}

// Warp-wide best candidate, in lane 0 (and, with `all`, broadcast to every lane).
__device__ __forceinline__ PivotCand cand_warp_reduce(PivotCand a, bool all)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        cand_merge(a, cand_shfl_down(a, off));
    if (all) {
        a.key = __shfl_sync(0xFFFFFFFFu, a.key, 0);
        a.val = __shfl_sync(0xFFFFFFFFu, a.val, 0);
        a.row = __shfl_sync(0xFFFFFFFFu, a.row, 0);
        a.slot = __shfl_sync(0xFFFFFFFFu, a.slot, 0);
    }
    return a;
}

__global__ void __launch_bounds__(PANEL1_THREADS) lu_panel_cluster_kernel(uint32_t *__restrict__ P, size_t lda,
                                                                          int M, int jb, int R, int row0,
                                                                          int *__restrict__ ipiv,
                                                                          int *__restrict__ info)
{
    namespace cgs = cooperative_groups;
    cgs::cluster_group cluster = cgs::this_cluster();
    const int rank = (int)cluster.block_rank(), ncta = (int)cluster.num_blocks();
    extern __shared__ __align__(16) double s_rows[]; // [R][jb][T]: this CTA's slots, FP64
    __shared__ PivotCand s_wc[2][32];                // each warp's candidate, by column parity
    __shared__ double s_u[PANEL1_MAX_JB];            // -u_kc of the current pivot row
    __shared__ PivotInfo s_pi;
    __shared__ uint32_t s_tab[F64_CONST_ENTRIES]; // rounding constants (F64ConstTable)
    if (*info < 0) // written only by earlier launches: the same in every CTA
        return;
    const int T = (int)blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wpc = T >> 5;
    for (int i = tid; i < F64_CONST_ENTRIES; i += T)
        s_tab[i] = f64_round_const_top(i);
    const F64ConstTable cof{s_tab}; // read only after the first barrier below
    auto own = [&](int r, int c) -> double & { return s_rows[((size_t)r * jb + c) * T + tid]; };
    int row[PANEL1_MAX_R]; // the logical row each slot holds (-1: none)
#pragma unroll
    for (int r = 0; r < PANEL1_MAX_R; ++r) {
        const int i = (r * T + tid) * ncta + rank;
        row[r] = (r < R && i < M) ? i : -1;
        if (row[r] >= 0)
            for (int c = 0; c < jb; ++c)
                own(r, c) = p32_to_double(P[i + (size_t)c * lda]);
    }
    const int nslots = ncta * wpc;
    for (int k = 0; k < jb; ++k) {
        PivotCand cand = {-2.0, 0.0, -1, 0};
#pragma unroll
        for (int r = 0; r < PANEL1_MAX_R; ++r)
            if (row[r] >= k) {
                const double v = own(r, k);
                cand_merge(cand, PivotCand{pivot_key(v), v, row[r], (r << 16) | (rank << 10) | tid});
            }
        cand = cand_warp_reduce(cand, false);
        if (lane == 0)
            s_wc[k & 1][warp] = cand;
        panel_sync(cluster, ncta); // the warps' candidates, cluster-wide
        cand = PivotCand{-2.0, 0.0, -1, 0};
        for (int s = lane; s < nslots; s += 32)
            cand_merge(cand, *cluster.map_shared_rank(&s_wc[k & 1][s % wpc], s / wpc));
        cand = cand_warp_reduce(cand, true);
        const int p = cand.row;
        const uint32_t piv = p32_from_double_exact(cand.val);
        // u from the pivot row's slot (after the interchange it is row k)
        const int sr = cand.slot >> 16, sq = (cand.slot >> 10) & 63, st = cand.slot & 1023;
        double *src = cluster.map_shared_rank(s_rows, sq) + (size_t)sr * jb * T + st;
        for (int c = k + 1 + tid; c < jb; c += T)
            s_u[c] = -src[(size_t)c * T];
        if (tid == T - 1) {
            PivotInfo pi;
            pi.row = p;
            pi.piv = piv;
            if (piv == 0) {
                pi.mode = 0;
                pi.recip = 0;
                if (rank == 0 && *info == 0)
                    *info = row0 + k + 1;
            } else if ((int32_t)pabs(piv) >= (int32_t)1u) { // |pivot| >= sfmin = FLT_MIN -> minpos
                pi.mode = 1;
                pi.recip = pdiv_est(P32_ONE, piv);
            } else {
                pi.mode = 2; // NaR pivot: element-wise division (Rgetrf2.cpp:124-126)
                pi.recip = 0;
            }
            if (rank == 0)
                ipiv[row0 + k] = row0 + p + 1; // 1-based, global
            s_pi = pi;
        }
        if (p != k) {
            if (piv == 0) {
                // A zero pivot leaves its own column in place (Rgetrf2.cpp:107-117) while the
                // recursion's Rlaswp calls move rows k and p in every other column: the two
                // slots trade their column-k values back.  Only row k's holder touches them
                // (the pivot's slot is read above at columns > k only).
#pragma unroll
                for (int r = 0; r < PANEL1_MAX_R; ++r)
                    if (row[r] == k) {
                        src[(size_t)k * T] = own(r, k);
                        own(r, k) = cand.val;
                    }
            }
#pragma unroll
            for (int r = 0; r < PANEL1_MAX_R; ++r)
                row[r] = row[r] == k ? p : (row[r] == p ? k : row[r]);
        }
        __syncthreads(); // u and the scaling decision
        const PivotInfo pi = s_pi;
        const double drecip = p32_to_double(pi.recip);
#pragma unroll
        for (int r = 0; r < PANEL1_MAX_R; ++r) {
            if (row[r] > k) {
                double *rw = &own(r, 0);
                // Rscal (x*recip, the FP64 product step) or the element-wise division
                const double dl = pi.mode == 1 ? f64_posit_mul_checked(rw[(size_t)k * T], drecip, cof)
                                               : p32_to_double(lu_scaled(p32_from_double_exact(rw[(size_t)k * T]), pi));
                rw[(size_t)k * T] = dl;
                for (int c = k + 1; c < jb; ++c) // a_ic + (-u_kc)*l_i in the FP64 step
                    rw[(size_t)c * T] = f64_posit_mac_checked(rw[(size_t)c * T], s_u[c], dl, cof);
            }
        }
    }
    panel_sync(cluster, ncta); // no CTA leaves while another may still read its shared memory
#pragma unroll
    for (int r = 0; r < PANEL1_MAX_R; ++r)
        if (row[r] >= 0)
            for (int c = 0; c < jb; ++c)
                P[row[r] + (size_t)c * lda] = p32_from_double_exact(own(r, c));
}

// After a panel of columns [j, j+jb) (jb <= ROWS_JB_MAX): the panel's row interchanges
// (Rlaswp, Rlaswp.cpp:77-107, in ascending order) on every column outside the panel, and
// the unit-lower solve of the U12 block (Rtrsm('L', 'L', 'N', 'U'), Rtrsm.cpp:139-154, zero
// multipliers skipped as there) on the columns right of it, in one launch: one warp per
// column, lane i holding row j+i and (for an interchange with a row below the block) that
// row's value, loaded together; the interchanges run in order as exchanges between lanes,
// the solve as jb steps of one multiply-add per lane with the step's b_k from its lane.
constexpr int ROWS_JB_MAX = 32;
constexpr int ROWS_THREADS = 256; // 8 columns per block

__global__ void __launch_bounds__(ROWS_THREADS) lu_rows_kernel(uint32_t *__restrict__ A, size_t lda, int n, int j,
                                                               int jb, const int *__restrict__ ipiv)
{
    constexpr unsigned FULL = 0xFFFFFFFFu;
    __shared__ double s_L[ROWS_JB_MAX * ROWS_JB_MAX]; // l_ik at [i * ROWS_JB_MAX + k], FP64
    __shared__ int s_t[ROWS_JB_MAX];                  // interchange i: row j+i <-> row s_t[i] (0-based)
    __shared__ int s_alias[ROWS_JB_MAX];              // below the block: the first interchange with that row
    const int tid = threadIdx.x, lane = tid & 31;
    for (int e = tid; e < jb * jb; e += ROWS_THREADS) {
        const int i = e % jb, k = e / jb;
        s_L[i * ROWS_JB_MAX + k] = p32_to_double(A[(j + i) + (size_t)(j + k) * lda]);
    }
    for (int i = tid; i < jb; i += ROWS_THREADS)
        s_t[i] = ipiv[j + i] - 1;
    __syncthreads();
    for (int i = tid; i < jb; i += ROWS_THREADS) {
        int a = -1;
        if (s_t[i] >= j + jb) {
            a = i;
            for (int q = 0; q < i; ++q)
                if (s_t[q] == s_t[i]) {
                    a = q;
                    break;
                }
        }
        s_alias[i] = a;
    }
    __syncthreads();
    const int ci = blockIdx.x * (ROWS_THREADS / 32) + (tid >> 5);
    if (ci >= n - jb)
        return; // the whole warp
    const int c = ci < j ? ci : ci + jb; // the columns outside the panel
    uint32_t *col = A + (size_t)c * lda;
    const bool row = lane < jb;
    const int my_t = row ? s_t[lane] : 0, my_alias = row ? s_alias[lane] : -1;
    uint32_t v = row ? col[j + lane] : 0u;               // row j+lane
    uint32_t w = (my_alias == lane) ? col[my_t] : 0u;  // row my_t (below the block)
    for (int i = 0; i < jb; ++i) {
        const int t = s_t[i];
        if (t == j + i)
            continue;
        const bool in = t < j + jb;
        const int o = in ? t - j : s_alias[i];
        const uint32_t vi = __shfl_sync(FULL, v, i);
        const uint32_t vo = __shfl_sync(FULL, in ? v : w, o);
        if (lane == o) {
            if (in)
                v = vi;
            else
                w = vi;
        }
        if (lane == i)
            v = vo;
    }
    if (my_alias == lane)
        col[my_t] = w;
    if (c > j) { // U12 <- L11^-1 A12, column-oriented as Rtrsm.cpp:139-154 (unit diagonal)
        double x = row ? p32_to_double(v) : 0.0;
        for (int k = 0; k < jb; ++k) {
            const double bk = __shfl_sync(FULL, x, k);
            if (bk != 0.0 && lane > k && row)
                x = f64_posit_mac_checked(x, -bk, s_L[lane * ROWS_JB_MAX + k]);
        }
        v = p32_from_double(x);
    }
    if (row)
        col[j + lane] = v;
}

// ---------------------------------------------------------------------------
// Rlaswp (Rlaswp.cpp:77-107): interchanges k1..k2 (1-based, global ipiv) applied in order
// to `ncols` columns starting at A; one thread per column.
// ---------------------------------------------------------------------------
__global__ void laswp_kernel(uint32_t *__restrict__ A, size_t lda, int ncols, int k1, int k2,
                             const int *__restrict__ ipiv, int incx, const int *__restrict__ info)
{
    if (info && *info < 0)
        return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols)
        return;
    uint32_t *col = A + (size_t)c * lda;
    if (incx > 0) {
        for (int i = k1; i <= k2; ++i) {
            int ip = ipiv[i - 1];
            if (ip != i) {
                uint32_t t = col[i - 1];
                col[i - 1] = col[ip - 1];
                col[ip - 1] = t;
            }
        }
    } else {
        for (int i = k2; i >= k1; --i) {
            int ip = ipiv[i - 1];
            if (ip != i) {
                uint32_t t = col[i - 1];
                col[i - 1] = col[ip - 1];
                col[ip - 1] = t;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Triangular solves with many right-hand sides: one CTA per column of B, one thread per
// row (strided), the column in shared memory.  Loop orders and zero skips as in
// Rtrsm.cpp:115-156 (side = L, trans = N).
// ---------------------------------------------------------------------------
// lower, unit or non-unit diagonal: forward substitution (Rtrsm.cpp:139-154).  The column
// is held in shared memory as FP64 (posit32 values are exact there) and every update
// b_i - b_k*a_ik is the FP64 multiply-add step of the GEMM (posit32.cuh, f64_posit_mac),
// its rare flagged steps redone on patterns.  NaR travels as NaN (every step that meets
// it is flagged and redone on patterns, which give NaR).
PG_HD double trsm_update(double c, double t, double a) { return f64_posit_mac_checked(c, t, a); }

// The column: staged in shared memory as FP64, or (too long for that) left in place as
// patterns and converted at every access.
template <bool STAGED>
struct SolveCol {
    double *s;
    uint32_t *g;
    __device__ double get(int i) const { return STAGED ? s[i] : p32_to_double(g[i]); }
    __device__ void set(int i, double v) const
    {
        if (STAGED)
            s[i] = v;
        else
            g[i] = p32_from_double(v);
    }
};

template <bool STAGED>
__global__ void trsm_lln_kernel(const uint32_t *__restrict__ L, size_t ldl, uint32_t *__restrict__ B, size_t ldb,
                                int m, bool unit, const int *__restrict__ info)
{
    extern __shared__ double s_x[];
    if (info && *info < 0)
        return;
    uint32_t *bcol = B + (size_t)blockIdx.x * ldb;
    const SolveCol<STAGED> x{s_x, bcol};
    if (STAGED)
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            s_x[i] = p32_to_double(bcol[i]);
    __syncthreads();
    for (int k = 0; k < m; ++k) {
        double bk = x.get(k);
        if (bk != 0.0) {
            if (!unit) {
                bk = p32_to_double(pdiv_est(p32_from_double(bk), L[k + (size_t)k * ldl]));
                __syncthreads();
                if (threadIdx.x == 0)
                    x.set(k, bk);
            }
            const double nb = -bk;
            const uint32_t *lk = L + (size_t)k * ldl;
            for (int i = k + 1 + threadIdx.x; i < m; i += blockDim.x)
                x.set(i, trsm_update(x.get(i), nb, p32_to_double(lk[i])));
        }
        __syncthreads();
    }
    if (STAGED)
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            bcol[i] = p32_from_double(s_x[i]);
}

// upper, non-unit diagonal: backward substitution (Rtrsm.cpp:121-136), as above
template <bool STAGED>
__global__ void trsm_lun_kernel(const uint32_t *__restrict__ U, size_t ldu, uint32_t *__restrict__ B, size_t ldb,
                                int m, bool unit, const int *__restrict__ info)
{
    extern __shared__ double s_x[];
    if (info && *info < 0)
        return;
    uint32_t *bcol = B + (size_t)blockIdx.x * ldb;
    const SolveCol<STAGED> x{s_x, bcol};
    if (STAGED)
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            s_x[i] = p32_to_double(bcol[i]);
    __syncthreads();
    for (int k = m - 1; k >= 0; --k) {
        double bk = x.get(k);
        if (bk != 0.0) {
            if (!unit) {
                bk = p32_to_double(pdiv_est(p32_from_double(bk), U[k + (size_t)k * ldu]));
                __syncthreads();
                if (threadIdx.x == 0)
                    x.set(k, bk);
            }
            const double nb = -bk;
            const uint32_t *uk = U + (size_t)k * ldu;
            for (int i = threadIdx.x; i < k; i += blockDim.x)
                x.set(i, trsm_update(x.get(i), nb, p32_to_double(uk[i])));
        }
        __syncthreads();
    }
    if (STAGED)
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            bcol[i] = p32_from_double(s_x[i]);
}

// The same two solves with the column staged in shared memory and each thread's rows of
// the triangle's next column loaded into registers while the current step runs, so no step
// waits for memory: rows tid + j*T (j < J) belong to thread tid.  The thread that holds the
// next step's row divides it by its diagonal right after that row's last update, before the
// step's barrier, so every thread reads b_k already divided: one division per step instead
// of one per thread, and one barrier per step.
template <bool UPPER, int J>
__global__ void __launch_bounds__(1024) trsm_col_kernel(const uint32_t *__restrict__ A, size_t lda,
                                                        uint32_t *__restrict__ B, size_t ldb, int m, bool unit,
                                                        const int *__restrict__ info)
{
    extern __shared__ double s_x[];
    if (info && *info < 0)
        return;
    uint32_t *bcol = B + (size_t)blockIdx.x * ldb;
    const int T = (int)blockDim.x, tid = threadIdx.x;
    for (int i = tid; i < m; i += T)
        s_x[i] = p32_to_double(bcol[i]);
    auto step_col = [&](int st) { return UPPER ? m - 1 - st : st; };
    uint32_t lc[J], ln[J]; // this thread's rows of the current / next column
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int i = tid + j * T;
        lc[j] = i < m ? A[i + (size_t)step_col(0) * lda] : 0u;
    }
    // b_i / a_ii by the thread holding row i (Rtrsm.cpp:127, 145; b_i = 0 is left alone, as
    // the reference skips it)
    auto finish = [&](int i, uint32_t d) {
        const double v = s_x[i];
        if (!unit && v != 0.0)
            s_x[i] = p32_to_double(pdiv_est(p32_from_double_exact(v), d));
    };
    uint32_t dn = unit ? 0u : A[step_col(0) + (size_t)step_col(0) * lda];
    __syncthreads(); // the column is staged
    if (tid == step_col(0) % T)
        finish(step_col(0), dn);
    __syncthreads();
    for (int st = 0; st < m; ++st) {
        const int k = step_col(st), kn = step_col(st + 1);
        if (st + 1 < m) {
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int i = tid + j * T;
                ln[j] = i < m ? A[i + (size_t)kn * lda] : 0u;
            }
            if (!unit)
                dn = A[kn + (size_t)kn * lda];
        }
        const double bk = s_x[k]; // final: divided by its row's thread at the end of the last step
        if (bk != 0.0) {          // zero multipliers skipped (Rtrsm.cpp:125-126, 143-144)
            const double nb = -bk;
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int i = tid + j * T;
                if (UPPER ? i < k : (i > k && i < m))
                    s_x[i] = trsm_update(s_x[i], nb, p32_to_double(lc[j]));
            }
        }
        // the next step's row has had its last update: its thread divides it now
        if (st + 1 < m && tid == kn % T)
            finish(kn, dn);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < J; ++j)
            lc[j] = ln[j];
    }
    for (int i = tid; i < m; i += T)
        bcol[i] = p32_from_double_exact(s_x[i]);
}

template <bool UPPER>
static cudaError_t launch_col(int J, int nrhs, int threads, const uint32_t *A, size_t lda, uint32_t *B, size_t ldb,
                              int m, bool unit, const int *info, cudaStream_t st)
{
    const size_t bytes = (size_t)m * sizeof(double);
    const void *fn = J <= 1 ? (const void *)trsm_col_kernel<UPPER, 1>
                   : J <= 2 ? (const void *)trsm_col_kernel<UPPER, 2>
                   : J <= 4 ? (const void *)trsm_col_kernel<UPPER, 4>
                   : J <= 8 ? (const void *)trsm_col_kernel<UPPER, 8>
                            : (const void *)trsm_col_kernel<UPPER, 16>;
    if (bytes > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess)
            return e;
    }
    void *args[] = {(void *)&A, (void *)&lda, (void *)&B, (void *)&ldb, (void *)&m, (void *)&unit, (void *)&info};
    return cudaLaunchKernel(fn, dim3((unsigned)nrhs), dim3((unsigned)threads), args, bytes, st);
}

// Forward / backward solve launches: staged when the column fits in shared memory (with
// the prefetching kernel up to 16 rows per thread).
static cudaError_t launch_lln(int nrhs, int threads, const uint32_t *L, size_t ldl, uint32_t *B, size_t ldb,
                              int m, bool unit, const int *info, cudaStream_t st)
{
    const size_t bytes = (size_t)m * sizeof(double);
    const int J = (m + threads - 1) / threads;
    if (bytes <= 227 * 1024 && J <= 16) {
        const cudaError_t e = launch_col<false>(J, nrhs, threads, L, ldl, B, ldb, m, unit, info, st);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (bytes <= 227 * 1024) {
        if (bytes > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(trsm_lln_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)bytes);
            if (e != cudaSuccess)
                return e;
        }
        trsm_lln_kernel<true><<<nrhs, threads, bytes, st>>>(L, ldl, B, ldb, m, unit, info);
    } else {
        trsm_lln_kernel<false><<<nrhs, threads, 0, st>>>(L, ldl, B, ldb, m, unit, info);
    }
    return cudaGetLastError();
}

static cudaError_t launch_lun(int nrhs, int threads, const uint32_t *U, size_t ldu, uint32_t *B, size_t ldb,
                              int m, bool unit, const int *info, cudaStream_t st)
{
    const size_t bytes = (size_t)m * sizeof(double);
    const int J = (m + threads - 1) / threads;
    if (bytes <= 227 * 1024 && J <= 16) {
        const cudaError_t e = launch_col<true>(J, nrhs, threads, U, ldu, B, ldb, m, unit, info, st);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (bytes <= 227 * 1024) {
        if (bytes > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(trsm_lun_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)bytes);
            if (e != cudaSuccess)
                return e;
        }
        trsm_lun_kernel<true><<<nrhs, threads, bytes, st>>>(U, ldu, B, ldb, m, unit, info);
    } else {
        trsm_lun_kernel<false><<<nrhs, threads, 0, st>>>(U, ldu, B, ldb, m, unit, info);
    }
    return cudaGetLastError();
}

// Lower, transposed (Rtrsm.cpp:175-186): one block per right-hand side; the column is
// staged in shared memory (when it fits) and one thread runs the whole dependent chain
// (trsm_chain.cuh).
constexpr int LLT_SMEM_MAX = 227 * 1024;

__global__ void __launch_bounds__(32) trsm_llt_kernel(const uint32_t *__restrict__ L, size_t ldl,
                                                      uint32_t *__restrict__ B, size_t ldb, int m, bool staged,
                                                      bool unit, bool upper, const int *__restrict__ info)
{
    extern __shared__ uint32_t s_col[];
    if (info && *info != 0) // a factorization stopped before this solve
        return;
    uint32_t *bcol = B + (size_t)blockIdx.x * ldb;
    if (!staged) {
        if (threadIdx.x == 0)
            llt_chain(L, ldl, bcol, m, unit, upper);
        return;
    }
    for (int i = threadIdx.x; i < m; i += 32)
        s_col[i] = bcol[i];
    __syncwarp();
    if (threadIdx.x == 0)
        llt_chain(L, ldl, s_col, m, unit, upper);
    __syncwarp();
    for (int i = threadIdx.x; i < m; i += 32)
        bcol[i] = s_col[i];
}

// The dot-form solves split over warps (below): the scan form's window parameters.
constexpr int LLT_SCAN_E = 4;
constexpr int LLT_SHORT_WINDOW = 64; // a window that ends sooner ...
constexpr int LLT_SEQ_STEPS = 32;    // ... is followed by this many sequential steps

// Term storage: FP64, or (for long columns) the posit32 patterns of the products.
template <class T>
struct LltTerms;
template <>
struct LltTerms<double> {
    using View = TermsF64;
    __device__ static double store(uint32_t p) { return p32_to_double(p); }
};
template <>
struct LltTerms<uint32_t> {
    using View = TermsP32;
    __device__ static uint32_t store(uint32_t p) { return p; }
};

// ---------------------------------------------------------------------------
// The dot-form solve with the row's windows spread over a group of warps.
// ---------------------------------------------------------------------------
// Rtrsm('L', 'L', 'T'), Rtrsm.cpp:175-186: for i = m-1 down to 0, t = b_i, t = t - a_ki*b_k
// for k = i+1 .. m-1 in order, b_i = t / a_ii (UPPER: Rtrsm('L', 'U', 'T'),
// Rtrsm.cpp:160-173, rows in increasing order, terms k = 0 .. i-1; the warps scan the terms
// k <= i-2, computed while row i-1 ran, then add the last one from the value just
// finished).  One block of 2 * LLT_GROUP_WARPS warps per right-hand side: the first
// LLT_GROUP_WARPS warps (the consumer group) sum each row in windows of
// LLT_GROUP_WARPS * 32 * LLT_SCAN_E terms in the scan form (trsm_chain.cuh) -- the first term
// (the b just finished) by one exact step -- while the others compute the next row's terms
// -a_k * b_k (all whose b_k are final) into the other half of a double buffer.  A
// window is the warp scan of step maps in every consumer warp, then each warp's composed map
// goes to shared memory, a named barrier (the consumer group only), each warp composes the
// maps of the warps before it with its own exclusive prefix and walks its addends, each warp
// reports its first step the scan form does not cover, a named barrier, and every consumer
// thread takes the first such step of the window (or the window's end value).  Every
// consumer thread then holds the same running value; the exact steps and the sequential
// runs after a window cut short run in every consumer thread alike (no broadcast needed).
constexpr int LLT_GROUP_WARPS = 4;
constexpr int LLT_GROUP_THREADS = 2 * LLT_GROUP_WARPS * 32;

// One window's exchange between the consumer warps; two of them, used by turns, so that a
// window's results may be read while the next window's are written.
struct __align__(16) GroupScan {
    SegFn wt[LLT_GROUP_WARPS];     // each consumer warp's composed map
    int jbad[LLT_GROUP_WARPS];     // each warp's first uncovered step (-1: none)
    int32_t Mbad[LLT_GROUP_WARPS]; // M before that step
    int32_t Mend;                  // M after the window's last addend
};
static_assert(LLT_GROUP_WARPS == 4, "the window's results are read as int4 vectors");

__device__ __forceinline__ void group_bar() { asm volatile("bar.sync 1, %0;" ::"r"(LLT_GROUP_WARPS * 32) : "memory"); }

template <int E, class Q>
__device__ double group_chain_scan(double t, Q q, int pos, int end, GroupScan *gsb, int &turn)
{
    constexpr unsigned FULL = 0xFFFFFFFFu;
    const int ct = threadIdx.x, lane = ct & 31, w = ct >> 5;
    while (pos < end) {
        GroupScan *gs = gsb + turn;
        SegParams sp;
        if (!seg_begin(t, sp)) { // zero, or outside the fast window: one exact step
            t = chain_add_one(t, q[pos]);
            ++pos;
            continue;
        }
        const int wend = min(end, pos + LLT_GROUP_WARPS * 32 * E);
        const int j0 = pos + ct * E;
        SegFn fe[E];
        int32_t K[E];
        bool rk[E];
        SegFn f = {0, 0};
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double qv = j0 + e < wend ? q[j0 + e] : 0.0; // 0 is the identity map
            fe[e] = seg_fn(qv, sp, K[e], rk[e]);
            f = seg_then(f, fe[e]);
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            SegFn o;
            o.c0 = __shfl_up_sync(FULL, f.c0, off);
            o.c1 = __shfl_up_sync(FULL, f.c1, off);
            if (lane >= off)
                f = seg_then(o, f);
        }
        SegFn ex;
        ex.c0 = __shfl_up_sync(FULL, f.c0, 1);
        ex.c1 = __shfl_up_sync(FULL, f.c1, 1);
        if (lane == 0)
            ex = SegFn{0, 0};
        if (lane == 31)
            gs->wt[w] = f;
        group_bar();
        const int4 wt01 = *reinterpret_cast<const int4 *>(&gs->wt[0]);
        const int4 wt23 = *reinterpret_cast<const int4 *>(&gs->wt[2]);
        SegFn pre = {0, 0};
        if (w > 0)
            pre = SegFn{wt01.x, wt01.y};
        if (w > 1)
            pre = seg_then(pre, SegFn{wt01.z, wt01.w});
        if (w > 2)
            pre = seg_then(pre, SegFn{wt23.x, wt23.y});
        int32_t M = seg_apply(seg_then(pre, ex), sp.M0);
        int jbad = -1;
        int32_t Mbad = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const bool live = (jbad < 0) & (j0 + e < wend);
            const bool ok = seg_valid(M, K[e], rk[e], sp);
            if (live & !ok) {
                jbad = j0 + e;
                Mbad = M;
            }
            if (live & ok)
                M = seg_apply(fe[e], M);
        }
        const unsigned bal = __ballot_sync(FULL, jbad >= 0);
        if (bal == 0) {
            if (lane == 0)
                gs->jbad[w] = -1;
        } else if (lane == __ffs(bal) - 1) {
            gs->jbad[w] = jbad;
            gs->Mbad[w] = Mbad;
        }
        if (ct == (wend - 1 - pos) / E) // the thread holding the window's last addend
            gs->Mend = M;
        group_bar();
        // the first warp's first uncovered step (warps hold increasing positions)
        const int4 jb4 = *reinterpret_cast<const int4 *>(gs->jbad);
        const int4 mb4 = *reinterpret_cast<const int4 *>(gs->Mbad);
        const int32_t Me = gs->Mend;
        int js = jb4.w;
        int32_t Ms = mb4.w;
        if (jb4.z >= 0) { js = jb4.z; Ms = mb4.z; }
        if (jb4.y >= 0) { js = jb4.y; Ms = mb4.y; }
        if (jb4.x >= 0) { js = jb4.x; Ms = mb4.x; }
        // The next window writes the other exchange; this one is written again only after
        // the next window's first group barrier, which every consumer reaches after the
        // reads above.
        turn ^= 1;
        if (js < 0) {
            t = sp.us * (double)Me;
            pos = wend;
        } else {
            t = chain_add_one(sp.us * (double)Ms, q[js]);
            const bool cut_short = js - pos < LLT_SHORT_WINDOW;
            pos = js + 1;
            if (cut_short) {
                const int cnt = min(LLT_SEQ_STEPS, end - pos);
                t = chain_add_run_reg(t, q + pos, cnt);
                pos += cnt;
            }
        }
    }
    return t;
}

template <class T, bool UPPER = false>
__global__ void __launch_bounds__(LLT_GROUP_THREADS) trsm_ltx_group_kernel(const uint32_t *__restrict__ L,
                                                                           size_t ldl, uint32_t *__restrict__ B,
                                                                           size_t ldb, int m, bool unit,
                                                                           const int *__restrict__ info)
{
    extern __shared__ __align__(16) unsigned char smem_pc[];
    T *s_q = reinterpret_cast<T *>(smem_pc); // [2][m]: terms
    uint32_t *s_b = reinterpret_cast<uint32_t *>(s_q + 2 * (size_t)m);
    __shared__ uint32_t s_nar[2];
    __shared__ GroupScan s_gs[2];
    if (info && *info != 0) // a factorization stopped before this solve
        return;
    uint32_t *bcol = B + (size_t)blockIdx.x * ldb;
    const int tid = threadIdx.x;
    constexpr int NC = LLT_GROUP_WARPS * 32; // consumer threads
    for (int k = tid; k < m; k += LLT_GROUP_THREADS)
        s_b[k] = bcol[k];
    if (tid < 2)
        s_nar[tid] = 0;
    __syncthreads();
    uint32_t xprev = 0; // the row finished last, b_{i+1} (lower) or b_{i-1} (upper) (consumers)
    int turn = 0;       // which of s_gs the next window uses (consumers)
    for (int step = 0; step < m; ++step) {
        const int i = UPPER ? step : m - 1 - step;
        const int cur = step & 1;
        if (tid < NC) {
            const uint32_t *li = L + (size_t)i * ldl;
            const uint32_t bi = s_b[i];
            uint32_t nar = (bi == P32_NAR) | s_nar[cur];
            double c = p32_to_double(bi == P32_NAR ? 0u : bi);
            const typename LltTerms<T>::View q{s_q + (size_t)cur * m};
            if (!UPPER && i + 1 < m) {
                c = chain_add_one(c, llt_term(li[i + 1], xprev, &nar));
                c = group_chain_scan<LLT_SCAN_E>(c, q, i + 2, m, s_gs, turn);
            }
            if (UPPER && i >= 1) {
                c = group_chain_scan<LLT_SCAN_E>(c, q, 0, i - 1, s_gs, turn);
                c = chain_add_one(c, llt_term(li[i - 1], xprev, &nar));
            }
            uint32_t t = nar ? P32_NAR : p32_from_double(c);
            if (!unit)
                t = pdiv_est(t, li[i]);
            xprev = t;
            group_bar(); // every consumer has read s_nar[cur]
            if (tid == 0) {
                s_b[i] = t;
                s_nar[cur] = 0;
            }
        } else if (step + 1 < m) {
            // the terms of the next row whose b_k are final: k = i+1 .. m-1 of row i-1
            // (lower), k = 0 .. i-1 of row i+1 (upper)
            const int nxt = UPPER ? i + 1 : i - 1;
            const int kbeg = UPPER ? 0 : i + 1, kend = UPPER ? i : m;
            const uint32_t *lp = L + (size_t)nxt * ldl;
            T *qn = s_q + (size_t)(cur ^ 1) * m;
            uint32_t nar = 0;
            for (int k = kbeg + (tid - NC); k < kend; k += LLT_GROUP_THREADS - NC) {
                const uint32_t p = pmul(0u - s_b[k], lp[k]); // (-b)*a == -(a*b) bit for bit
                nar |= p == P32_NAR;
                qn[k] = LltTerms<T>::store(p == P32_NAR ? 0u : p);
            }
            if (nar)
                s_nar[cur ^ 1] = 1;
        }
        __syncthreads();
    }
    for (int k = tid; k < m; k += LLT_GROUP_THREADS)
        bcol[k] = s_b[k];
}

size_t llt_pc_smem_bytes(int m, size_t term_bytes) { return (size_t)m * (2 * term_bytes + 4); }

// ---------------------------------------------------------------------------
// Cholesky panel (lower)
// ---------------------------------------------------------------------------
// Two launches per panel column k, as for LU:
//   chol_update_kernel  blocks over (rows > k) x (column groups in (k, jb)): l_ik =
//                       (1/l_kk)*a_ik for the rows below the diagonal block (those of the
//                       block were scaled by the diagonal step; Rtrsm.cpp:265-268), then
//                       a_ic += (-l_ck)*l_ik for k < c <= i.  Column k is only read; the
//                       first column group writes the new l_ik to a scratch column.
//   chol_diag_kernel    one block: the scratch column into column k, then the diagonal step
//                       of column k+1: l_kk = sqrt(a_kk) -- a_kk <= 0 in posit order, NaR
//                       included, stops with info (Rpotrf2.cpp:90-93) -- and
//                       l_ck = (1/l_kk)*a_ck for the rows c in (k, jb).
struct CholSync {
    uint32_t recip; // 1/l_kk of the current column
};

__global__ void chol_diag_kernel(uint32_t *__restrict__ P, size_t lda, int M, int jb, int k, int row0,
                                 int *__restrict__ info, CholSync *__restrict__ sync,
                                 const uint32_t *__restrict__ lcol, int copy_col)
{
    __shared__ uint32_t s_recip;
    __shared__ int s_stop;
    if (*info != 0)
        return;
    if (copy_col >= 0) {
        uint32_t *pc = P + (size_t)copy_col * lda;
        for (int r = (copy_col + 1 > jb ? copy_col + 1 : jb) + threadIdx.x; r < M; r += blockDim.x)
            pc[r] = lcol[r];
    }
    if (k >= jb)
        return;
    uint32_t *pk = P + (size_t)k * lda;
    if (threadIdx.x == 0) {
        uint32_t akk = pk[k];
        s_stop = (int32_t)akk <= 0;
        if (s_stop) {
            *info = row0 + k + 1;
        } else {
            uint32_t lkk = psqrt_est(akk);
            s_recip = pdiv_est(P32_ONE, lkk);
            pk[k] = lkk;
            sync->recip = s_recip;
        }
    }
    __syncthreads();
    if (s_stop)
        return;
    for (int c = k + 1 + threadIdx.x; c < jb; c += blockDim.x)
        pk[c] = pmul(s_recip, pk[c]);
}

__global__ void __launch_bounds__(PANEL_ROWS) chol_update_kernel(uint32_t *__restrict__ P, size_t lda, int M,
                                                                 int jb, int k, const int *__restrict__ info,
                                                                 const CholSync *__restrict__ sync,
                                                                 uint32_t *__restrict__ lcol)
{
    __shared__ double s_l[PANEL_CG]; // -l_ck for this block's columns, FP64
    if (*info != 0)
        return;
    const uint32_t recip = sync->recip;
    const uint32_t *pk = P + (size_t)k * lda;
    const int c0 = k + 1 + blockIdx.y * PANEL_CG;
    if (threadIdx.x < PANEL_CG && c0 + (int)threadIdx.x < jb)
        s_l[threadIdx.x] = -p32_to_double(pk[c0 + threadIdx.x]); // scaled by the diagonal step
    __syncthreads();
    const int i = k + 1 + blockIdx.x * PANEL_ROWS + threadIdx.x;
    if (i >= M)
        return;
    const uint32_t a = pk[i];
    const uint32_t l = i >= jb ? pmul(recip, a) : a;
    if (blockIdx.y == 0 && i >= jb)
        lcol[i] = l;
    const double dl = p32_to_double(l);
    const int cn = min(min(PANEL_CG, jb - c0), i - c0 + 1);
    for (int j = 0; j < cn; ++j) { // a_ic + (-l_ck)*l_i in the FP64 step (posit32.cuh)
        uint32_t *pc = P + i + (size_t)(c0 + j) * lda;
        *pc = p32_from_double_exact(f64_posit_mac_checked(p32_to_double(*pc), s_l[j], dl));
    }
}

// Lower Cholesky panel in one thread-block cluster, held in shared memory (rows dealt out
// as in lu_panel_cluster_kernel; here they never change places), the counterpart of
// chol_diag_kernel + chol_update_kernel.  The thread holding row k forms l_kk and 1/l_kk
// (Rpotrf2.cpp:90-97) right after its own update of column k-1 and writes the decision and
// 1/l_kk into every CTA.  Per column: a cluster barrier (A); every thread scales its rows
// below the diagonal (Rtrsm.cpp:265-268), the holders of the diagonal block's rows also
// writing their -l_ck into every CTA; a cluster barrier (B); each thread updates its rows.
// With one CTA the barriers are the block's.  A failed diagonal (info) ends the loop in
// every CTA at the same column; the rows are written back either way.
__global__ void __launch_bounds__(PANEL1_THREADS) chol_panel_cluster_kernel(uint32_t *__restrict__ P, size_t lda,
                                                                            int M, int jb, int R, int row0,
                                                                            int *__restrict__ info)
{
    namespace cgs = cooperative_groups;
    cgs::cluster_group cluster = cgs::this_cluster();
    const int rank = (int)cluster.block_rank(), ncta = (int)cluster.num_blocks();
    extern __shared__ __align__(16) double s_rows[]; // [R][jb][T]: this CTA's rows, FP64
    __shared__ double s_l[PANEL1_MAX_JB];           // -l_ck of the current column
    __shared__ uint32_t s_recip;                    // 1/l_kk
    __shared__ int s_stop;                          // a_kk <= 0 or NaR
    __shared__ uint32_t s_tab[F64_CONST_ENTRIES];   // rounding constants (F64ConstTable)
    if (*info != 0) // written only by earlier launches: the same in every CTA
        return;
    const int T = (int)blockDim.x, tid = threadIdx.x;
    for (int i = tid; i < F64_CONST_ENTRIES; i += T)
        s_tab[i] = f64_round_const_top(i);
    const F64ConstTable cof{s_tab}; // read only after the first barrier below
    auto own = [&](int r, int c) -> double & { return s_rows[((size_t)r * jb + c) * T + tid]; };
    auto row_of = [&](int r) { return (r * T + tid) * ncta + rank; };
    for (int r = 0; r < R; ++r) {
        const int i = row_of(r);
        if (i < M)
            for (int c = 0; c < jb; ++c)
                own(r, c) = p32_to_double(P[i + (size_t)c * lda]);
    }
    // From the holder of row k: l_kk in place, the decision and 1/l_kk into every CTA.
    auto diag = [&](int r, int k) {
        const uint32_t akk = p32_from_double_exact(own(r, k));
        const int stop = (int32_t)akk <= 0; // NaR included (Rpotrf2.cpp:90-93)
        uint32_t recip = 0;
        if (!stop) {
            const uint32_t lkk = psqrt_est(akk);
            own(r, k) = p32_to_double(lkk);
            recip = pdiv_est(P32_ONE, lkk);
        }
        for (int q = 0; q < ncta; ++q) {
            *cluster.map_shared_rank(&s_stop, q) = stop;
            *cluster.map_shared_rank(&s_recip, q) = recip;
        }
    };
    panel_sync(cluster, ncta); // every CTA has started: distributed shared memory may be written
    for (int r = 0; r < R; ++r)
        if (row_of(r) == 0)
            diag(r, 0);
    for (int k = 0; k < jb; ++k) {
        panel_sync(cluster, ncta); // A: the decision and 1/l_kk; every read of the last column's -l_ck done
        if (s_stop) { // the same in every CTA
            // written only here, after every CTA has passed its entry check of *info
            if (rank == 0 && tid == 0)
                *info = row0 + k + 1;
            break;
        }
        const double drecip = p32_to_double(s_recip);
        for (int r = 0; r < R; ++r) {
            const int i = row_of(r);
            if (i > k && i < M) { // (1/l_kk)*a_ik, the FP64 product step
                const double l = f64_posit_mul_checked(own(r, k), drecip, cof);
                own(r, k) = l;
                if (i < jb)
                    for (int q = 0; q < ncta; ++q)
                        *cluster.map_shared_rank(&s_l[i], q) = -l;
            }
        }
        panel_sync(cluster, ncta); // B: the column's -l_ck in every CTA
        for (int r = 0; r < R; ++r) {
            const int i = row_of(r);
            if (i > k && i < M) {
                double *rw = &own(r, 0);
                const double dl = rw[(size_t)k * T];
                const int cend = min(jb - 1, i);
                for (int c = k + 1; c <= cend; ++c) // a_ic + (-l_ck)*l_i in the FP64 step
                    rw[(size_t)c * T] = f64_posit_mac_checked(rw[(size_t)c * T], s_l[c], dl, cof);
                if (i == k + 1 && i < jb) // the next diagonal, from its holder's own update
                    diag(r, k + 1);
            }
        }
    }
    panel_sync(cluster, ncta); // no CTA leaves while another may still write its shared memory
    for (int r = 0; r < R; ++r) {
        const int i = row_of(r);
        if (i < M)
            for (int c = 0; c < jb; ++c)
                P[i + (size_t)c * lda] = p32_from_double_exact(own(r, c));
    }
}

// ---------------------------------------------------------------------------
// Upper Cholesky diagonal block: Rpotrf2('U') (Rpotrf2.cpp:86-131) in one CTA
// ---------------------------------------------------------------------------
// The recursion exactly as the reference runs it, since the upper factor's bits depend on
// how the work is grouped: a 1x1 block takes the square root (a <= 0, NaR included, stops
// with info); a larger one splits n1 = n/2, n2 = n - n1, factors A11, solves
// A12 <- U11^-T A12 (Rtrsm('L', 'U', 'T', 'N'), Rtrsm.cpp:160-173: per column, for each
// row i, t = b_i, t = t - u_ki*b_k over k < i in order, b_i = t / u_ii), updates
// A22 <- -(A12^T A12) + A22 on and above the diagonal (Rsyrk('U', 'T'), Rsyrk.cpp:182-195:
// each entry's dot product summed from zero in order, then alpha*t + beta*c) and factors
// A22.  The recursion runs on an explicit stack in shared memory; the solves are one
// thread per column, the update one thread per entry, with barriers in between.
constexpr int POTRF2_CTA_THREADS = 256;
constexpr int POTRF2_CTA_MAX = 128; // larger blocks recurse on the host with many-block kernels

__global__ void __launch_bounds__(POTRF2_CTA_THREADS) potrf2_upper_cta_kernel(uint32_t *__restrict__ A, size_t lda,
                                                                              int n, int row0, int *__restrict__ info)
{
    constexpr int DEPTH = 16;
    __shared__ int s_off[DEPTH], s_n[DEPTH], s_stage[DEPTH];
    __shared__ int s_sp, s_stop;
    if (*info != 0)
        return;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_sp = 1;
        s_off[0] = 0;
        s_n[0] = n;
        s_stage[0] = 0;
        s_stop = 0;
    }
    __syncthreads();
    for (;;) {
        const int sp = s_sp;
        if (sp == 0)
            break;
        const int off = s_off[sp - 1], nn = s_n[sp - 1], stage = s_stage[sp - 1];
        __syncthreads(); // the frame is read before thread 0 changes the stack
        if (nn == 1) {
            if (tid == 0) {
                uint32_t *d = A + off + (size_t)off * lda;
                const uint32_t a = *d;
                if ((int32_t)a <= 0) { // Rpotrf2.cpp:90-93 (NaR is below zero in posit order)
                    *info = row0 + off + 1;
                    s_stop = 1;
                } else {
                    *d = psqrt_est(a);
                }
                s_sp = sp - 1;
            }
        } else {
            const int n1 = nn / 2, n2 = nn - n1;
            uint32_t *a11 = A + off + (size_t)off * lda;
            uint32_t *a12 = A + off + (size_t)(off + n1) * lda;
            uint32_t *a22 = A + (off + n1) + (size_t)(off + n1) * lda;
            if (stage == 0) {
                if (tid == 0) {
                    s_stage[sp - 1] = 1;
                    s_off[sp] = off;
                    s_n[sp] = n1;
                    s_stage[sp] = 0;
                    s_sp = sp + 1;
                }
            } else if (stage == 1) {
                for (int j = tid; j < n2; j += POTRF2_CTA_THREADS) { // A12 <- U11^-T A12
                    uint32_t *b = a12 + (size_t)j * lda;
                    for (int i = 0; i < n1; ++i) {
                        const uint32_t *ui = a11 + (size_t)i * lda;
                        double t = p32_to_double(b[i]);
                        for (int k = 0; k < i; ++k)
                            t = f64_posit_mac_checked(t, -p32_to_double(b[k]), p32_to_double(ui[k]));
                        b[i] = pdiv_est(p32_from_double(t), ui[i]);
                    }
                }
                __syncthreads();
                const int cnt = n2 * (n2 + 1) / 2; // A22 <- -(A12^T A12) + A22, i <= j
                for (int e = tid; e < cnt; e += POTRF2_CTA_THREADS) {
                    int j = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f); // e = j(j+1)/2 + i
                    while (j * (j + 1) / 2 > e)
                        --j;
                    while ((j + 1) * (j + 2) / 2 <= e)
                        ++j;
                    const int i = e - j * (j + 1) / 2;
                    const uint32_t *ci = a12 + (size_t)i * lda, *cj = a12 + (size_t)j * lda;
                    double t = 0.0;
                    for (int l = 0; l < n1; ++l)
                        t = f64_posit_mac_checked(t, p32_to_double(ci[l]), p32_to_double(cj[l]));
                    uint32_t *c = a22 + i + (size_t)j * lda;
                    *c = padd(pmul(0xC0000000u /* -1 */, p32_from_double(t)), pmul(P32_ONE, *c));
                }
                __syncthreads();
                if (tid == 0) {
                    s_stage[sp - 1] = 2;
                    s_off[sp] = off + n1;
                    s_n[sp] = n2;
                    s_stage[sp] = 0;
                    s_sp = sp + 1;
                }
            } else if (tid == 0) {
                s_sp = sp - 1;
            }
        }
        __syncthreads();
        if (s_stop)
            return;
    }
}

// ---------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

// Panel width for an n x n factorization when the caller passes nb <= 0: the widths the
// autotuner (posit_gpu_b200/autotune.py) measured fastest on B200, by size bucket.  LU and
// lower Cholesky give the same bits at every width.
int tuned_panel_width(bool lu, int n)
{
    struct Row {
        int n, lu, chol;
    };
    static const Row rows[] = {{0, 24, 16},    {512, 24, 24},  {1024, 24, 16},   {2048, 24, 24},
                               {4096, 32, 32}, {8192, 32, 24}, {16384, 128, 128}};
    int nb = 16;
    for (const Row &r : rows)
        if (n >= r.n)
            nb = lu ? r.lu : r.chol;
    return nb;
}

size_t rgetrf_workspace_bytes(int m, int n, int nb)
{
    int mn = imin(m, n);
    if (nb < 1)
        nb = 1;
    int jb = imin(nb, mn);
    size_t g = mn > jb ? gemm_workspace_bytes(m - jb > 0 ? m - jb : 1, n - jb > 0 ? n - jb : 1, jb) : 0;
    return panel_ws_bytes(m) + g;
}

// The panel form: the cluster panel held in shared memory when its rows fit (ncta CTAs,
// one per PANEL1_ROWS_PER_CTA rows up to 8, T threads each -- the CTA's rows rounded up to
// whole warps, at most 1024 -- R slots per thread, R * jb * T FP64 values of shared memory
// at most 24 * 1024), else the two-launch form (ncta = 0).
struct PanelForm {
    int ncta, R, T; // CTAs (0: the panel does not fit), slots per thread, threads per CTA
};
static PanelForm panel_form(int M, int jb, int max_ctas)
{
    if (jb > PANEL1_MAX_JB)
        return {0, 0, 0};
    const int cap = max_ctas > 0 ? std::min(max_ctas, PANEL1_MAX_CTAS) : PANEL1_MAX_CTAS;
    const int ncta = std::max(1, std::min(cap, (M + PANEL1_ROWS_PER_CTA - 1) / PANEL1_ROWS_PER_CTA));
    const int rpc = (M + ncta - 1) / ncta; // rows per CTA
    const int T = std::min(PANEL1_THREADS, (rpc + 31) / 32 * 32), R = (rpc + T - 1) / T;
    if ((size_t)R * jb * T > (size_t)PANEL1_SMEM_ENTRIES * PANEL1_THREADS || R > PANEL1_MAX_R)
        return {0, 0, 0};
    return {ncta, R, T};
}

template <class... Args>
static cudaError_t launch_panel_cluster(void (*kernel)(Args...), PanelForm f, int jb, cudaStream_t st, Args... args)
{
    const size_t smem = (size_t)f.R * jb * f.T * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         PANEL1_SMEM_ENTRIES * PANEL1_THREADS * (int)sizeof(double));
    if (e != cudaSuccess)
        return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)f.ncta);
    cfg.blockDim = dim3((unsigned)f.T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)f.ncta;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

static dim3 panel_grid(int M, int jb, int k)
{
    return dim3((unsigned)imax((M - k - 1 + PANEL_ROWS - 1) / PANEL_ROWS, 1),
                (unsigned)imax((jb - k - 1 + PANEL_CG - 1) / PANEL_CG, 1));
}

// Rgetrf.cpp:95-132 with the device kernels above.  `ws` holds the pivot record, the
// scratch column and the trailing GEMM's workspace.
cudaError_t rgetrf_launch(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info, void *ws,
                          cudaStream_t st, int max_ctas)
{
    const int mn = imin(m, n);
    if (nb < 1)
        nb = 1;
    PivotInfo *pinfo = reinterpret_cast<PivotInfo *>(ws);
    uint32_t *lcol = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(ws) + 256);
    void *gws = reinterpret_cast<unsigned char *>(ws) + panel_ws_bytes(m);
    const size_t L = (size_t)lda;
    for (int j = 0; j < mn; j += nb) {
        const int jb = imin(mn - j, nb);
        const int M = m - j;
        uint32_t *P = A + j + (size_t)j * L;
        uint32_t *lc = lcol + j; // indexed by panel-local row
        const PanelForm pf = panel_form(M, jb, max_ctas);
        if (pf.ncta > 0) {
            cudaError_t e = launch_panel_cluster(lu_panel_cluster_kernel, pf, jb, st, P, L, M, jb, pf.R, j, ipiv, info);
            if (e != cudaSuccess)
                return e;
        } else {
            lu_pivot_kernel<<<1, 1024, 0, st>>>(P, L, M, jb, 0, j, ipiv, info, pinfo, lc, -1);
            for (int k = 0; k < jb; ++k) {
                lu_update_kernel<<<panel_grid(M, jb, k), PANEL_ROWS, 0, st>>>(P, L, M, jb, k, info, pinfo, lc);
                lu_pivot_kernel<<<1, 1024, 0, st>>>(P, L, M, jb, k + 1, j, ipiv, info, pinfo, lc, k);
            }
        }
        if (jb <= ROWS_JB_MAX) {
            if (n > jb)
                lu_rows_kernel<<<(n - jb + ROWS_THREADS / 32 - 1) / (ROWS_THREADS / 32), ROWS_THREADS, 0, st>>>(
                    A, L, n, j, jb, ipiv);
        } else {
            if (j > 0)
                laswp_kernel<<<(j + 127) / 128, 128, 0, st>>>(A, L, j, j + 1, j + jb, ipiv, 1, info);
            if (j + jb < n) {
                const int nr = n - j - jb;
                laswp_kernel<<<(nr + 127) / 128, 128, 0, st>>>(A + (size_t)(j + jb) * L, L, nr, j + 1, j + jb, ipiv,
                                                              1, info);
                cudaError_t e = launch_lln(nr, 256, P, L, A + j + (size_t)(j + jb) * L, L, jb, true, info, st);
                if (e != cudaSuccess)
                    return e;
            }
        }
        if (j + jb < n) {
            const int nr = n - j - jb;
            uint32_t *A12 = A + j + (size_t)(j + jb) * L;
            cudaError_t e = cudaSuccess;
            if (j + jb < m) {
                e = gemm_launch(true, true, m - j - jb, nr, jb, 0xC0000000u /* -1 */,
                                            A + (j + jb) + (size_t)j * L, lda, A12, lda, P32_ONE,
                                            A + (j + jb) + (size_t)(j + jb) * L, lda, gws, st);
                if (e != cudaSuccess)
                    return e;
            }
        }
    }
    return cudaGetLastError();
}

size_t rpotrf_workspace_bytes(int n, int nb)
{
    if (nb < 1)
        nb = 1;
    int jb = imin(nb, n);
    return panel_ws_bytes(n) + (n > jb ? gemm_workspace_bytes(n - jb, n - jb, jb) : 0);
}

// Lower Cholesky (Rpotrf.cpp:124-142 / Rpotrf2.cpp:132-146 order, blocked right-looking).
cudaError_t rpotrf_lower_launch(int n, uint32_t *A, int lda, int nb, int *info, void *ws, cudaStream_t st,
                                int max_ctas)
{
    if (nb < 1)
        nb = 1;
    CholSync *sync = reinterpret_cast<CholSync *>(ws);
    uint32_t *lcol = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(ws) + 256);
    void *gws = reinterpret_cast<unsigned char *>(ws) + panel_ws_bytes(n);
    const size_t L = (size_t)lda;
    for (int j = 0; j < n; j += nb) {
        const int jb = imin(n - j, nb);
        const int M = n - j;
        uint32_t *P = A + j + (size_t)j * L;
        uint32_t *lc = lcol + j;
        const PanelForm pf = panel_form(M, jb, max_ctas);
        if (pf.ncta > 0) {
            cudaError_t e = launch_panel_cluster(chol_panel_cluster_kernel, pf, jb, st, P, L, M, jb, pf.R, j, info);
            if (e != cudaSuccess)
                return e;
        } else {
            chol_diag_kernel<<<1, 256, 0, st>>>(P, L, M, jb, 0, j, info, sync, lc, -1);
            for (int k = 0; k < jb; ++k) {
                chol_update_kernel<<<panel_grid(M, jb, k), PANEL_ROWS, 0, st>>>(P, L, M, jb, k, info, sync, lc);
                chol_diag_kernel<<<1, 256, 0, st>>>(P, L, M, jb, k + 1, j, info, sync, lc, k);
            }
        }
        if (j + jb < n) {
            const int nr = n - j - jb;
            const uint32_t *L21 = A + (j + jb) + (size_t)j * L;
            cudaError_t e = gemm_launch_lower(true, false, nr, nr, jb, 0xC0000000u /* -1 */, L21, lda, L21,
                                              lda, P32_ONE, A + (j + jb) + (size_t)(j + jb) * L, lda, gws, st, info);
            if (e != cudaSuccess)
                return e;
        }
    }
    return cudaGetLastError();
}

// Upper Cholesky (Rpotrf.cpp:96-118): left-looking and blocked by nb in the reference's
// order, which the upper factor's bits depend on.  For each block column j: the diagonal
// block's update by the rows above it (Rsyrk('U', 'T'): the TN GEMM on its upper
// triangle), its factorization (Rpotrf2('U'), recursive), the block row's update (Rgemm
// 'T', 'N') and solve (Rtrsm('L', 'U', 'T', 'N')).  nb <= 1 or nb >= n is Rpotrf2 on the
// whole matrix (Rpotrf.cpp:86-91).  Kernels after a failed diagonal do nothing.
static cudaError_t launch_ltx(bool upper, bool unit, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B,
                              int ldb, const int *info, cudaStream_t st);

static void potrf2_upper_plan(int n, size_t *ws)
{
    if (n <= POTRF2_CTA_MAX)
        return;
    const int n1 = n / 2, n2 = n - n1;
    potrf2_upper_plan(n1, ws);
    *ws = std::max(*ws, gemm_workspace_bytes(n2, n2, n1));
    potrf2_upper_plan(n2, ws);
}

size_t rpotrf_upper_workspace_bytes(int n, int nb)
{
    size_t ws = 0;
    if (nb <= 1 || nb >= n) {
        potrf2_upper_plan(n, &ws);
        return ws;
    }
    for (int j = 0; j < n; j += nb) {
        const int jb = imin(nb, n - j);
        if (j > 0) {
            ws = std::max(ws, gemm_workspace_bytes(jb, jb, j));
            if (j + jb < n)
                ws = std::max(ws, gemm_workspace_bytes(jb, n - j - jb, j));
        }
        potrf2_upper_plan(jb, &ws);
    }
    return ws;
}

static cudaError_t potrf2_upper(uint32_t *A, int lda, int off, int n, int *info, void *ws, cudaStream_t st)
{
    const size_t L = (size_t)lda;
    if (n <= POTRF2_CTA_MAX) {
        potrf2_upper_cta_kernel<<<1, POTRF2_CTA_THREADS, 0, st>>>(A + off + (size_t)off * L, L, n, off, info);
        return cudaGetLastError();
    }
    const int n1 = n / 2, n2 = n - n1;
    cudaError_t e = potrf2_upper(A, lda, off, n1, info, ws, st);
    if (e == cudaSuccess)
        e = launch_ltx(true, false, n1, n2, A + off + (size_t)off * L, lda, A + off + (size_t)(off + n1) * L, lda,
                       info, st);
    if (e == cudaSuccess)
        e = gemm_launch_tri(TRI_UPPER, false, true, n2, n2, n1, 0xC0000000u /* -1 */,
                            A + off + (size_t)(off + n1) * L, lda, A + off + (size_t)(off + n1) * L, lda, P32_ONE,
                            A + (off + n1) + (size_t)(off + n1) * L, lda, ws, st, info);
    if (e == cudaSuccess)
        e = potrf2_upper(A, lda, off + n1, n2, info, ws, st);
    return e;
}

cudaError_t rpotrf_upper_launch(int n, uint32_t *A, int lda, int nb, int *info, void *ws, cudaStream_t st)
{
    if (nb <= 1 || nb >= n)
        return potrf2_upper(A, lda, 0, n, info, ws, st);
    const size_t L = (size_t)lda;
    for (int j = 0; j < n; j += nb) {
        const int jb = imin(nb, n - j);
        cudaError_t e = cudaSuccess;
        if (j > 0) // Rsyrk('U', 'T', jb, j, -1, A(0:j, j:j+jb), 1, A(j:j+jb, j:j+jb))
            e = gemm_launch_tri(TRI_UPPER, false, true, jb, jb, j, 0xC0000000u /* -1 */, A + (size_t)j * L, lda,
                                A + (size_t)j * L, lda, P32_ONE, A + j + (size_t)j * L, lda, ws, st, info);
        if (e == cudaSuccess)
            e = potrf2_upper(A, lda, j, jb, info, ws, st);
        if (e == cudaSuccess && j + jb < n) {
            const int nr = n - j - jb;
            if (j > 0) // Rgemm('T', 'N', jb, nr, j, -1, A(0:j, j:j+jb), A(0:j, j+jb:n), 1, A(j:j+jb, j+jb:n))
                e = gemm_launch_tri(TRI_FULL, false, true, jb, nr, j, 0xC0000000u /* -1 */, A + (size_t)j * L, lda,
                                    A + (size_t)(j + jb) * L, lda, P32_ONE, A + j + (size_t)(j + jb) * L, lda, ws, st,
                                    info);
            if (e == cudaSuccess) // Rtrsm('L', 'U', 'T', 'N', jb, nr, 1, A(j:j+jb, j:j+jb), A(j:j+jb, j+jb:n))
                e = launch_ltx(true, false, jb, nr, A + j + (size_t)j * L, lda, A + j + (size_t)(j + jb) * L, lda,
                               info, st);
        }
        if (e != cudaSuccess)
            return e;
    }
    return cudaGetLastError();
}

// Rgetrs.cpp:84-114 (trans = 'N'): interchanges, L (unit) forward, U backward.
cudaError_t rgetrs_launch(int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb,
                          cudaStream_t st)
{
    const int threads = 1024;
    laswp_kernel<<<(nrhs + 127) / 128, 128, 0, st>>>(B, ldb, nrhs, 1, n, ipiv, 1, nullptr);
    cudaError_t e = launch_lln(nrhs, threads, A, lda, B, ldb, n, true, nullptr, st);
    if (e == cudaSuccess)
        e = launch_lun(nrhs, threads, A, lda, B, ldb, n, false, nullptr, st);
    return e;
}

// The dot-form solves with the triangle transposed: L^-T B (Rtrsm('L', 'L', 'T'),
// Rtrsm.cpp:175-186) or, with `upper`, U^-T B (Rtrsm('L', 'U', 'T'), Rtrsm.cpp:160-173).
// One block per right-hand side: the scan-form kernel where its terms fit in shared
// memory (FP64 where 20n bytes fit, patterns where 12n do), else one thread's chain.
// A nonzero *info (when given) turns the solve into a no-op.
static cudaError_t launch_ltx(bool upper, bool unit, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B,
                              int ldb, const int *info, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    const size_t pc8 = llt_pc_smem_bytes(n, sizeof(double)), pc4 = llt_pc_smem_bytes(n, sizeof(uint32_t));
    if (pc8 <= (size_t)LLT_SMEM_MAX || pc4 <= (size_t)LLT_SMEM_MAX) {
        const bool f64 = pc8 <= (size_t)LLT_SMEM_MAX;
        const size_t pc = f64 ? pc8 : pc4;
        const void *fn = f64 ? (upper ? (const void *)trsm_ltx_group_kernel<double, true>
                                      : (const void *)trsm_ltx_group_kernel<double, false>)
                             : (upper ? (const void *)trsm_ltx_group_kernel<uint32_t, true>
                                      : (const void *)trsm_ltx_group_kernel<uint32_t, false>);
        if (pc > 48 * 1024) {
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pc);
            if (e != cudaSuccess)
                return e;
        }
        if (f64 && upper)
            trsm_ltx_group_kernel<double, true><<<nrhs, LLT_GROUP_THREADS, pc, st>>>(A, lda, B, ldb, n, unit, info);
        else if (f64)
            trsm_ltx_group_kernel<double, false><<<nrhs, LLT_GROUP_THREADS, pc, st>>>(A, lda, B, ldb, n, unit, info);
        else if (upper)
            trsm_ltx_group_kernel<uint32_t, true><<<nrhs, LLT_GROUP_THREADS, pc, st>>>(A, lda, B, ldb, n, unit, info);
        else
            trsm_ltx_group_kernel<uint32_t, false><<<nrhs, LLT_GROUP_THREADS, pc, st>>>(A, lda, B, ldb, n, unit, info);
        return cudaGetLastError();
    }
    const size_t col = (size_t)n * 4;
    const bool staged = col <= (size_t)LLT_SMEM_MAX;
    if (staged && col > 48 * 1024) {
        e = cudaFuncSetAttribute(trsm_llt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col);
        if (e != cudaSuccess)
            return e;
    }
    trsm_llt_kernel<<<nrhs, 32, staged ? col : 0, st>>>(A, lda, B, ldb, n, staged, unit, upper, info);
    return cudaGetLastError();
}

// Rpotrs.cpp:95-106 (uplo = 'L'): L forward, L^T backward.
cudaError_t rpotrs_lower_launch(int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb, cudaStream_t st)
{
    const int threads = 1024;
    cudaError_t e = launch_lln(nrhs, threads, A, lda, B, ldb, n, false, nullptr, st);
    if (e != cudaSuccess)
        return e;
    return launch_ltx(false, false, n, nrhs, A, lda, B, ldb, nullptr, st);
}

// Rpotrs.cpp:84-95 (uplo = 'U'): U^T forward (Rtrsm('L', 'U', 'T', 'N')), then U backward
// (Rtrsm('L', 'U', 'N', 'N')).
cudaError_t rpotrs_upper_launch(int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb, cudaStream_t st)
{
    cudaError_t e = launch_ltx(true, false, n, nrhs, A, lda, B, ldb, nullptr, st);
    if (e != cudaSuccess)
        return e;
    return launch_lun(nrhs, 1024, A, lda, B, ldb, n, false, nullptr, st);
}

// Rgetrs.cpp:99-113 (trans = 'T' or 'C'): U^T forward (non-unit), L^T backward (unit),
// then the interchanges applied in reverse order (Rlaswp with incx = -1).
cudaError_t rgetrs_trans_launch(int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb,
                                cudaStream_t st)
{
    cudaError_t e = launch_ltx(true, false, n, nrhs, A, lda, B, ldb, nullptr, st);
    if (e != cudaSuccess)
        return e;
    e = launch_ltx(false, true, n, nrhs, A, lda, B, ldb, nullptr, st);
    if (e != cudaSuccess)
        return e;
    laswp_kernel<<<(nrhs + 127) / 128, 128, 0, st>>>(B, ldb, nrhs, 1, n, ipiv, -1, nullptr);
    return cudaGetLastError();
}

} // namespace pg
