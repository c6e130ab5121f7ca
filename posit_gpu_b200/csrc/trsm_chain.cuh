// trsm_chain.cuh -- the transposed lower triangular solve of Rpotrs as one thread's chain.
//
// Rtrsm('L', 'L', 'T', 'N'), Rtrsm.cpp:175-186: for i = m-1 down to 0,
//     t = b_i;  t = t - a_ki * b_k  for k = i+1 .. m-1 (ascending);  b_i = t / a_ii.
// Each b_i's sum starts from the b_{i+1} just finished, so one right-hand side is a single
// chain of m(m-1)/2 dependent multiply-subtracts with two roundings each.  A thread owns one
// right-hand side and runs its whole chain with the accumulator held decoded; different
// right-hand sides are different threads.
//
// Latency is everything here.  Only the addition depends on the previous step: loads,
// decoding and the product of step k+1 can overlap the addition of step k, but not across
// a branch (a GPU issues in order and does not run past an unresolved branch).  So the
// steps run in blocks of CHAIN_BLOCK without a branch: the fast path's failure flags are
// OR-ed over the block and tested once at its end; in the rare block that has one, the
// block is replayed from its start value one exactly checked step at a time.  The next
// block's operands are loaded (clamped to stay in bounds) while the current one runs.
#pragma once
#include "posit32.cuh"

namespace pg {

constexpr int CHAIN_BLOCK = 8;

PG_HD dp32 chain_neg_b(uint32_t bk) { return decode_gemm_bf(bk == P32_NAR ? 0u : 0u - bk); }
PG_HD dp32 chain_a(uint32_t l) { return decode_gemm_bf(l == P32_NAR ? 0u : l); }

// b (this thread's right-hand side, m entries; shared or global memory) is overwritten
// with L^-T b.  L is read-only.  Host and device (the host build is what the CPU tests run).
PG_HD void llt_chain(const uint32_t *__restrict__ L, size_t ldl, uint32_t *b, int m, bool unit)
{
    constexpr int U = CHAIN_BLOCK;
    for (int i = m - 1; i >= 0; --i) {
        const uint32_t *li = L + (size_t)i * ldl; // column i of L: a_ki for k > i
        const uint32_t bi = b[i];                 // alpha*b with alpha == 1
        uint32_t nar = bi == P32_NAR;
        dp32 c = decode_gemm(nar ? 0u : bi);
        int k = i + 1;
        if (k + U <= m) {
            uint32_t lv[U], bv[U];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                lv[j] = li[k + j];
                bv[j] = b[k + j];
            }
            for (; k + U <= m; k += U) {
                // next block's operands (indexes clamped into [0, m))
                uint32_t ln[U], bn[U];
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    const int kk = k + U + j < m ? k + U + j : m - 1;
                    ln[j] = li[kk];
                    bn[j] = b[kk];
                }
                const dp32 c0 = c;
                uint32_t bad = 0;
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    // t - a_ki*b_k == t + (-b_k)*a_ki bit for bit: posit negation is exact
                    // and rounding is symmetric in sign.  NaR dominates
                    // (kernel_entry.cl:385-390, 414-417) and is carried in `nar`.
                    nar |= (lv[j] == P32_NAR) | (bv[j] == P32_NAR);
                    dp32 p, r;
                    uint32_t bm, ba;
                    dmul_core(chain_neg_b(bv[j]), chain_a(lv[j]), ComputedEntry{}, p, bm);
                    dadd_core(c, p, ComputedEntry{}, r, ba);
                    c = r;
                    bad |= bm | ba;
                }
                if (bad & 0x40000000u) {
                    c = c0;
                    for (int j = 0; j < U; ++j)
                        c = dmac_chain(c, chain_neg_b(bv[j]), chain_a(lv[j]));
                }
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    lv[j] = ln[j];
                    bv[j] = bn[j];
                }
            }
        }
        for (; k < m; ++k) {
            const uint32_t l = li[k], bk = b[k];
            nar |= (l == P32_NAR) | (bk == P32_NAR);
            c = dmac_chain(c, chain_neg_b(bk), chain_a(l));
        }
        uint32_t t = nar ? P32_NAR : encode(c);
        if (!unit)
            t = pdiv(t, li[i]);
        b[i] = t;
    }
}

// ---------------------------------------------------------------------------
// Split form: products computed elsewhere, the chain thread only adds.
// ---------------------------------------------------------------------------
// A decoded posit packed in 8 bytes (one shared-memory load): {scale, significand | sign<<31}.
struct alignas(8) PackedDp {
    int32_t s;
    uint32_t gx;
};
PG_HD PackedDp pack_q(const dp32 &d) { return PackedDp{d.s, d.g | (d.x << 31)}; }
PG_HD dp32 unpack_q(const PackedDp &p)
{
    dp32 d;
    d.s = p.s;
    d.g = p.gx & 0x7FFFFFFFu;
    d.x = p.gx >> 31;
    return d;
}

// The term -a_ki*b_k of the dot-form solve as the reference rounds it (p32_mul,
// kernel_entry.cl:399-538), decoded; *nar is set when it is NaR.
PG_HD PackedDp llt_term(uint32_t l, uint32_t bk, uint32_t *nar)
{
    const uint32_t p = pmul(0u - bk, l); // (-b)*a == -(a*b) bit for bit
    *nar |= p == P32_NAR;
    return pack_q(decode_gemm(p == P32_NAR ? 0u : p));
}

PG_HD_NOINLINE dp32 dadd_exact(dp32 c, dp32 q) { return decode_gemm(padd(encode(c), encode(q))); }

// c + q_0 + q_1 + ... + q_{count-1}, every addition rounded (p32_add), in that order; the
// q are decoded posit32 values.  Blocks of CHAIN_BLOCK additions without a branch, the
// failure flags tested per block, a flagged block replayed exactly.
PG_HD dp32 chain_add_run(dp32 c, const PackedDp *q, int count)
{
    constexpr int U = CHAIN_BLOCK;
    int k = 0;
    if (count >= U) {
        PackedDp v[U];
#pragma unroll
        for (int j = 0; j < U; ++j)
            v[j] = q[j];
        for (; k + U <= count; k += U) {
            PackedDp nv[U];
#pragma unroll
            for (int j = 0; j < U; ++j)
                nv[j] = q[k + U + j < count ? k + U + j : count - 1];
            const dp32 c0 = c;
            uint32_t bad = 0;
#pragma unroll
            for (int j = 0; j < U; ++j) {
                dp32 r;
                uint32_t ba;
                dadd_core(c, unpack_q(v[j]), ComputedEntry{}, r, ba);
                c = r;
                bad |= ba;
            }
            if (bad & 0x40000000u) {
                c = c0;
                for (int j = 0; j < U; ++j)
                    c = dadd_exact(c, unpack_q(v[j]));
            }
#pragma unroll
            for (int j = 0; j < U; ++j)
                v[j] = nv[j];
        }
    }
    for (; k < count; ++k) {
        const dp32 qk = unpack_q(q[k]);
        dp32 r;
        uint32_t ba;
        dadd_core(c, qk, ComputedEntry{}, r, ba);
        c = (ba & 0x40000000u) ? dadd_exact(c, qk) : r;
    }
    return c;
}

} // namespace pg
