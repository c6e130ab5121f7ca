// gemm_tile.cuh -- device pieces shared by the single-GEMM and the batched kernels:
// thread ownership inside a tile and the k-step loop.
#pragma once
#include "posit32.cuh"

namespace pg {

// Thread (tx, ty) owns rows {2tx, 2tx+1, 32+2tx, 33+2tx} and the same pattern of
// columns with ty: the 16-byte shared-memory loads of a warp then hit distinct banks.
__device__ __forceinline__ int own_off(int t, int q) { return (q >> 1) * 32 + 2 * t + (q & 1); }

// The k-steps of a tile in the FP64 form (posit32.cuh, f64_posit_mac): operands and
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
