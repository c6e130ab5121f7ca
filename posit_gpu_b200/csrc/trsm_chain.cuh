// trsm_chain.cuh -- the transposed lower triangular solve of Rpotrs as one thread's chain.
//
// Rtrsm('L', 'L', 'T', 'N'), Rtrsm.cpp:175-186: for i = m-1 down to 0,
//     t = b_i;  t = t - a_ki * b_k  for k = i+1 .. m-1 (ascending);  b_i = t / a_ii.
// Each b_i's sum starts from the b_{i+1} just finished, so one right-hand side is a single
// chain of m(m-1)/2 dependent multiply-subtracts with two roundings each.  A thread owns one
// right-hand side and runs its whole chain with the accumulator held decoded; different
// right-hand sides are different threads, so they cost no extra time.
#pragma once
#include "posit32.cuh"

namespace pg {

// b (this thread's right-hand side, m entries) is overwritten with L^-T b.  L is read-only.
__device__ __forceinline__ void llt_chain(const uint32_t *__restrict__ L, size_t ldl, uint32_t *b, int m, bool unit)
{
    for (int i = m - 1; i >= 0; --i) {
        const uint32_t *li = L + (size_t)i * ldl; // column i of L: a_ki for k > i
        const uint32_t bi = b[i];                 // alpha*b with alpha == 1
        uint32_t nar = bi == P32_NAR;
        dp32 c = decode_gemm(nar ? 0u : bi);
#pragma unroll 4
        for (int k = i + 1; k < m; ++k) {
            const uint32_t l = li[k], bk = b[k];
            nar |= (l == P32_NAR) | (bk == P32_NAR); // NaR dominates (kernel_entry.cl:385-390, 414-417)
            // t - a_ki*b_k == t + (-b_k)*a_ki bit for bit: posit negation is exact and
            // rounding is symmetric in sign
            const dp32 nb = decode_gemm(bk == P32_NAR ? 0u : 0u - bk);
            const dp32 a = decode_gemm(l == P32_NAR ? 0u : l);
            c = dmac_chain(c, nb, a);
        }
        uint32_t t = nar ? P32_NAR : encode(c);
        if (!unit)
            t = pdiv(t, li[i]);
        b[i] = t;
    }
}

} // namespace pg
