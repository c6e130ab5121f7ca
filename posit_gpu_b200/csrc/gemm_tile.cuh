// gemm_tile.cuh -- device pieces shared by the single-GEMM and the batched kernels:
// the packed decoded operand, thread ownership inside a tile, and the k-step loop.
#pragma once
#include "posit32.cuh"

namespace pg {

// ---------------------------------------------------------------------------
// Decoded element packing: {scale, significand | sign << 31}
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint2 pack_dp(const dp32 &d)
{
    return make_uint2((uint32_t)d.s, d.g | (d.x << 31));
}

__device__ __forceinline__ dp32 unpack_dp(uint32_t s, uint32_t gx)
{
    dp32 d;
    d.s = (int32_t)s;
    d.g = gx & 0x7FFFFFFFu;
    d.x = gx >> 31;
    return d;
}

// Thread (tx, ty) owns rows {2tx, 2tx+1, 32+2tx, 33+2tx} and the same pattern of
// columns with ty: the 16-byte shared-memory loads of a warp then hit distinct banks.
__device__ __forceinline__ int own_off(int t, int q) { return (q >> 1) * 32 + 2 * t + (q & 1); }

// `lmax` k-steps of a TM_ x TN_ register tile of accumulators over one staged pair of
// decoded tiles: as = [l][16*TM_] rows of op(A), ts = [l][16*TN_] columns of op(B).
// Each step is c <- c + t*a in the fast decoded path, committed branch-free; steps the
// fast path cannot do exactly are redone afterwards through the exact routines, in the
// same order, so the result is always the reference's.  Shared by the single-GEMM and
// the batched kernels.
template <int TM_, int TN_>
__device__ __forceinline__ void tile_steps(dp32 (&acc)[TM_][TN_], const uint2 *as, const uint2 *ts, int lmax,
                                           const RegimeEntry *tbl, int tx, int ty)
{
    constexpr int BM_ = 16 * TM_, BN_ = 16 * TN_;
    for (int l = 0; l < lmax; ++l) {
        dp32 a[TM_], t[TN_];
#pragma unroll
        for (int q = 0; q < TM_ / 2; ++q) {
            const uint4 v = *reinterpret_cast<const uint4 *>(as + l * BM_ + 32 * q + 2 * tx);
            a[2 * q] = unpack_dp(v.x, v.y);
            a[2 * q + 1] = unpack_dp(v.z, v.w);
        }
#pragma unroll
        for (int q = 0; q < TN_ / 2; ++q) {
            const uint4 v = *reinterpret_cast<const uint4 *>(ts + l * BN_ + 32 * q + 2 * ty);
            t[2 * q] = unpack_dp(v.x, v.y);
            t[2 * q + 1] = unpack_dp(v.z, v.w);
        }
        uint32_t fail = 0;
#pragma unroll
        for (int i = 0; i < TM_; ++i) {
#pragma unroll
            for (int j = 0; j < TN_; ++j) {
                dp32 p, r;
                uint32_t bm, ba;
                dmul_fast(t[j], a[i], tbl, p, bm);
                dadd_fast(acc[i][j], p, tbl, r, ba);
                // branch-free commit: a failed step leaves the accumulator as it was,
                // and sets bit i*TN_+j of `fail` (umulhi(2^30, 2^(idx+2)) = 2^idx)
                const uint32_t v = (bm | ba) & 0x40000000u;
                acc[i][j].s = v ? acc[i][j].s : r.s;
                acc[i][j].g = v ? acc[i][j].g : r.g;
                acc[i][j].x = v ? acc[i][j].x : r.x;
                fail += __umulhi(v, 4u << (i * TN_ + j));
            }
        }
        if (fail) { // rare: redo the failed steps exactly, in the same order
#pragma unroll
            for (int i = 0; i < TM_; ++i)
#pragma unroll
                for (int j = 0; j < TN_; ++j)
                    if (fail & (1u << (i * TN_ + j)))
                        acc[i][j] = dmac_exact(acc[i][j], t[j], a[i]);
        }
    }
}

// The same k-steps in the FP64 form (posit32.cuh, f64_posit_mac): operands and
// accumulators are posit32 values held in FP64; as = [l][16*TM_] and ts = [l][16*TN_] are
// FP64 tiles; ctab holds the rounding constants (F64ConstTable).  Failed steps are
// committed branch-free as no-ops and redone afterwards on patterns, in order.
template <int TM_, int TN_>
__device__ __forceinline__ void tile_steps_f64(double (&acc)[TM_][TN_], const double *as, const double *ts,
                                               int lmax, const uint32_t *ctab, int tx, int ty)
{
    constexpr int BM_ = 16 * TM_, BN_ = 16 * TN_;
    const F64ConstTable const_of{ctab};
    for (int l = 0; l < lmax; ++l) {
        double a[TM_], t[TN_];
#pragma unroll
        for (int q = 0; q < TM_ / 2; ++q) {
            const double2 v = *reinterpret_cast<const double2 *>(as + l * BM_ + 32 * q + 2 * tx);
            a[2 * q] = v.x;
            a[2 * q + 1] = v.y;
        }
#pragma unroll
        for (int q = 0; q < TN_ / 2; ++q) {
            const double2 v = *reinterpret_cast<const double2 *>(ts + l * BN_ + 32 * q + 2 * ty);
            t[2 * q] = v.x;
            t[2 * q + 1] = v.y;
        }
        uint32_t fail = 0;
#pragma unroll
        for (int i = 0; i < TM_; ++i) {
#pragma unroll
            for (int j = 0; j < TN_; ++j) {
                bool bad;
                const double r = f64_posit_mac(acc[i][j], t[j], a[i], const_of, bad);
                acc[i][j] = bad ? acc[i][j] : r;
                fail += __umulhi(bad ? 0x40000000u : 0u, 4u << (i * TN_ + j)); // 2^(i*TN_+j) when failed
            }
        }
        if (fail) { // rare: redo the failed steps exactly, in the same order
#pragma unroll
            for (int i = 0; i < TM_; ++i)
#pragma unroll
                for (int j = 0; j < TN_; ++j)
                    if (fail & (1u << (i * TN_ + j)))
                        acc[i][j] = f64_posit_mac_exact(acc[i][j], t[j], a[i]);
        }
    }
}

} // namespace pg
