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
// FP64 tiles; ctab holds the rounding constants (F64ConstTable).
//
// Two sets of accumulators take turns: step l reads one set and writes every result into
// the other, unconditionally, so the value before the step is still there when the step
// was flagged.  Only "was any step flagged" is kept on the fast path; in that (rare) case
// the step is evaluated again on the unchanged inputs -- the same flags come out -- and
// each flagged result is replaced by the exact step on patterns.  The order of the
// operations per accumulator is unchanged: one p32_mul and one p32_add per k, in k order.
template <int TM_, int TN_>
__device__ __forceinline__ void load_operands(const double *as, const double *ts, int l, int tx, int ty,
                                              double (&a)[TM_], double (&t)[TN_])
{
    constexpr int BM_ = 16 * TM_, BN_ = 16 * TN_;
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
}

// nxt = cur + t*a for every accumulator; true when any step was flagged.
template <int TM_, int TN_>
__device__ __forceinline__ bool step_all(const double (&cur)[TM_][TN_], double (&nxt)[TM_][TN_],
                                         const double (&a)[TM_], const double (&t)[TN_], F64ConstTable8 cof)
{
    bool any = false;
#pragma unroll
    for (int i = 0; i < TM_; ++i) {
#pragma unroll
        for (int j = 0; j < TN_; ++j) {
            bool bad;
            nxt[i][j] = f64_posit_mac(cur[i][j], t[j], a[i], cof, bad);
            any |= bad;
        }
    }
    return any;
}

// The flagged steps of step_all(cur -> nxt), found again and redone exactly.
template <int TM_, int TN_>
__device__ __forceinline__ void step_fixup(const double (&cur)[TM_][TN_], double (&nxt)[TM_][TN_],
                                           const double (&a)[TM_], const double (&t)[TN_], F64ConstTable8 cof)
{
#pragma unroll
    for (int i = 0; i < TM_; ++i) {
#pragma unroll
        for (int j = 0; j < TN_; ++j) {
            bool bad;
            (void)f64_posit_mac(cur[i][j], t[j], a[i], cof, bad);
            if (bad)
                nxt[i][j] = f64_posit_mac_exact(cur[i][j], t[j], a[i]);
        }
    }
}

template <int TM_, int TN_>
__device__ __forceinline__ void tile_steps_f64(double (&acc)[TM_][TN_], const double *as, const double *ts,
                                               int lmax, const double *ctab, int tx, int ty)
{
    const F64ConstTable8 cof{ctab};
    double alt[TM_][TN_];
    int l = 0;
    for (; l + 2 <= lmax; l += 2) {
        double a[TM_], t[TN_];
        load_operands<TM_, TN_>(as, ts, l, tx, ty, a, t);
        if (step_all<TM_, TN_>(acc, alt, a, t, cof))
            step_fixup<TM_, TN_>(acc, alt, a, t, cof);
        load_operands<TM_, TN_>(as, ts, l + 1, tx, ty, a, t);
        if (step_all<TM_, TN_>(alt, acc, a, t, cof))
            step_fixup<TM_, TN_>(alt, acc, a, t, cof);
    }
    if (l < lmax) { // odd tail: one step, then the result back into acc
        double a[TM_], t[TN_];
        load_operands<TM_, TN_>(as, ts, l, tx, ty, a, t);
        if (step_all<TM_, TN_>(acc, alt, a, t, cof))
            step_fixup<TM_, TN_>(acc, alt, a, t, cof);
#pragma unroll
        for (int i = 0; i < TM_; ++i)
#pragma unroll
            for (int j = 0; j < TN_; ++j)
                acc[i][j] = alt[i][j];
    }
}

} // namespace pg
