// trsm_chain.cuh -- the transposed lower triangular solve of Rpotrs: chains of dependent
// posit additions.
//
// Rtrsm('L', 'L', 'T', 'N'), Rtrsm.cpp:175-186: for i = m-1 down to 0,
//     t = b_i;  t = t - a_ki * b_k  for k = i+1 .. m-1 (ascending);  b_i = t / a_ii.
// Each b_i's sum starts from the b_{i+1} just finished, so one right-hand side is a single
// chain of m(m-1)/2 dependent multiply-subtracts with two roundings each.  Three forms:
//   * llt_chain: one thread runs a right-hand side's whole chain with the accumulator
//     held in the decoded integer form (the batched kernel; very long columns);
//   * chain_add_run / chain_add_run_reg: one thread's chain of additions in FP64, the
//     products computed elsewhere;
//   * the scan form (below): a warp sums a row's additions as a parallel prefix of step
//     maps on the posit grid (lapack.cu's transposed-solve kernel).
//
// For the one-thread chains latency is everything.  Only the addition depends on the previous step: loads,
// decoding and the product of step k+1 can overlap the addition of step k, but not across
// a branch (a GPU issues in order and does not run past an unresolved branch).  So the
// steps run in blocks of CHAIN_BLOCK without a branch: the fast path's failure flags are
// OR-ed over the block and tested once at its end; in the rare block that has one, the
// block is replayed from its start value one exactly checked step at a time.  The next
// block's operands are loaded (clamped to stay in bounds) while the current one runs.
#pragma once
#include "posit32.cuh"
#include "posit32_div.cuh"
#include <math.h>

namespace pg {

constexpr int CHAIN_BLOCK = 8;

PG_HD dp32 chain_neg_b(uint32_t bk) { return decode_dz_bf(bk == P32_NAR ? 0u : 0u - bk); }
PG_HD dp32 chain_a(uint32_t l) { return decode_dz_bf(l == P32_NAR ? 0u : l); }

// b (this thread's right-hand side, m entries; shared or global memory) is overwritten
// with L^-T b.  L is read-only.  Host and device (the host build is what the CPU tests run).
// With `upper`, the triangle is an upper one, U, and b is overwritten with U^-T b
// (Rtrsm('L', 'U', 'T'), Rtrsm.cpp:160-173): for i = 0 .. m-1, t = b_i, t = t - u_ki*b_k for
// k = 0 .. i-1 (ascending), b_i = t / u_ii -- the same chain run forwards.
PG_HD void llt_chain(const uint32_t *__restrict__ L, size_t ldl, uint32_t *b, int m, bool unit, bool upper = false)
{
    constexpr int U = CHAIN_BLOCK;
    for (int step = 0; step < m; ++step) {
        const int i = upper ? step : m - 1 - step;
        const uint32_t *li = L + (size_t)i * ldl; // column i: a_ki for k > i (lower) or k < i (upper)
        const uint32_t bi = b[i];                 // alpha*b with alpha == 1
        uint32_t nar = bi == P32_NAR;
        dp32 c = decode_dz(nar ? 0u : bi);
        int k = upper ? 0 : i + 1;
        const int kend = upper ? i : m;
        if (k + U <= kend) {
            uint32_t lv[U], bv[U];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                lv[j] = li[k + j];
                bv[j] = b[k + j];
            }
            for (; k + U <= kend; k += U) {
                // next block's operands (indexes clamped into [0, kend))
                uint32_t ln[U], bn[U];
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    const int kk = k + U + j < kend ? k + U + j : kend - 1;
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
        for (; k < kend; ++k) {
            const uint32_t l = li[k], bk = b[k];
            nar |= (l == P32_NAR) | (bk == P32_NAR);
            c = dmac_chain(c, chain_neg_b(bk), chain_a(l));
        }
        uint32_t t = nar ? P32_NAR : encode(c);
        if (!unit)
            t = pdiv_est(t, li[i]);
        b[i] = t;
    }
}

// ---------------------------------------------------------------------------
// Split form: products computed elsewhere, the chain thread only adds -- in FP64.
// ---------------------------------------------------------------------------
// A posit32 value is exact in FP64 (at most 28 significant bits, scale within +-120).
// One step t + q of the chain is then:
//   s = fl64(t + q)        exact whenever the operands' binades are at most 24 apart
//                          (the sum needs at most 29 + 24 bits);
//   r = (s + C) - C        C = 1.5 * 2^(e + 52 - fb), e the binade of s and fb the posit's
//                          fraction width there: round to nearest even at the posit's last
//                          fraction bit (ties to the even pattern, whose parity is the
//                          fraction's).
// The reference's p32_add is that rounding of the exact sum (within its 64-bit frame; an
// addend more than 30 binades down contributes nothing, which is also what rounding the
// exact sum gives).  More than 30 binades apart, fl64(t + q) may be inexact but lies far
// from every rounding boundary, so r is still right.  A step is handed to the exact path
// when the operands are 25..30 binades apart (the FP64 rounding could meet a posit tie),
// or when the sum's scale is outside the fast window (regime longer than 27 bits, fewer
// than one fraction bit; this includes an exactly cancelling sum, whose FP64 value is 0).
// The dependent path per step: three FP64 additions and a handful of integer operations
// that build C from the exponent of s.
// t + q rounded to posit32, both posit values held in FP64; bit 30 of `bad` is set when
// the step must come from the exact path instead.
PG_HD double f64_posit_add(double t, double q, uint32_t &bad)
{
    const double s = f64_add(t, q);
    const int32_t eb = (int32_t)((f64_bits(s) >> 52) & 0x7FF); // biased binade of s
    const int32_t k = (eb - 1023) >> 2;                         // regime value
    const int32_t run = (k ^ (k >> 31)) + 1;                     // regime run; fb = 28 - run
    const uint32_t hc = ((uint32_t)(eb + 24 + run) << 20) | 0x00080000u; // 1.5 * 2^(e - fb + 52)
    const double C = f64_from_bits((uint64_t)hc << 32);
    const double r = f64_add(f64_add(s, C), -C);
    // off the dependent path: is this step one the FP64 form does exactly?
    const int32_t et = (int32_t)((f64_bits(t) >> 52) & 0x7FF), eq = (int32_t)((f64_bits(q) >> 52) & 0x7FF);
    const int32_t gap = et > eq ? et - eq : eq - et;
    const bool risky = (et != 0) & (eq != 0) & (gap > 24) & (gap <= 30);
    const bool outside = (uint32_t)(eb - 1023 - FAST_LO) > (uint32_t)(FAST_HI - FAST_LO);
    bad |= (risky | outside) ? 0x40000000u : 0u;
    return r;
}

// The exact step on patterns (rare).
PG_HD double f64_posit_add_exact(double t, double q)
{
    return p32_to_double(padd(p32_from_double(t), p32_from_double(q)));
}

// The term -a_ki*b_k of the dot-form solve as the reference rounds it (p32_mul,
// kernel_entry.cl:399-538), in FP64; *nar is set when it is NaR (the term is then 0).
PG_HD double llt_term(uint32_t l, uint32_t bk, uint32_t *nar)
{
    const uint32_t p = pmul(0u - bk, l); // (-b)*a == -(a*b) bit for bit
    *nar |= p == P32_NAR;
    return p32_to_double(p == P32_NAR ? 0u : p);
}

// t + q_0 + q_1 + ... + q_{count-1}, every addition rounded (p32_add), in that order; t
// and the q are posit32 values in FP64.  (The kernels use the scan form and
// chain_add_run_reg below; this plain form is the sequence the tests hold them to.)
// Blocks of CHAIN_BLOCK steps without a branch, the flags tested once per block, a
// flagged block replayed exactly from its start.
PG_HD double chain_add_run(double t, const double *q, int count)
{
    constexpr int U = CHAIN_BLOCK;
    int k = 0;
    if (count >= U) {
        double v[U];
#pragma unroll
        for (int j = 0; j < U; ++j)
            v[j] = q[j];
        for (; k + U <= count; k += U) {
            double nv[U];
#pragma unroll
            for (int j = 0; j < U; ++j)
                nv[j] = q[k + U + j < count ? k + U + j : count - 1];
            const double t0 = t;
            uint32_t bad = 0;
#pragma unroll
            for (int j = 0; j < U; ++j)
                t = f64_posit_add(t, v[j], bad);
            if (bad & 0x40000000u) {
                t = t0;
                for (int j = 0; j < U; ++j)
                    t = f64_posit_add_exact(t, v[j]);
            }
#pragma unroll
            for (int j = 0; j < U; ++j)
                v[j] = nv[j];
        }
    }
    for (; k < count; ++k) {
        uint32_t bad = 0;
        const double r = f64_posit_add(t, q[k], bad);
        t = (bad & 0x40000000u) ? f64_posit_add_exact(t, q[k]) : r;
    }
    return t;
}


// ---------------------------------------------------------------------------
// Scan form: one row's chain of additions as a parallel prefix over the row.
// ---------------------------------------------------------------------------
// While the running value t stays in one binade [2^e, 2^(e+1)) with sign sg, it is an
// integer multiple M of the posit spacing u = 2^(e - fb) there (fb = the fraction width at
// scale e, M in [2^fb, 2^(fb+1))), and the fraction's last bit -- the pattern's last bit --
// is M's.  A step t + q with the exact sum inside that binade rounds (to nearest, ties to
// the even pattern) as
//     M' = M + K + [F > 1/2] + [F == 1/2] * ((M + K) & 1),   sg * q / u = K + F, 0 <= F < 1,
// which is p32_add's result (kernel_entry.cl:370-397): with the addend at most 30 binades
// down no bit of it leaves the reference's 64-bit frame, and a bit that falls below the
// sticky window after normalisation leaves set bits inside the window (the addend spans
// at most 28 bits), so the rounding decision is that of the exact sum; an addend further
// down has |K + F| < 1/8 and leaves M unchanged, as the reference does.  Steps 25..30
// binades down are still handed to the exact path, as the FP64 step does.
// The exact sum stays in the binade iff 2^fb <= M + K < 2^(fb+1).
//
// So a step is the map M -> M + c[M & 1] (c[0] and c[1] differ only on a tie), and such
// maps compose into maps of the same form.  A thread composes the maps of its slice of the
// row, an exclusive scan over the threads gives each slice its start, and each thread then
// walks its slice with the true M and reports the first step that leaves the binade (or
// starts at its top edge, or is risky).  All steps before that one are exact; the row
// goes on from there with one exact step and a new scan in the new binade.  A map's
// displacements saturate at +-SEG_SAT: only a path that has already left the binade can
// reach that, and no value past the first invalid step is used.
constexpr int32_t SEG_SAT = 1 << 29;

struct SegFn {
    int32_t c0, c1; // displacement for even / odd M
};

// Parameters of a run of steps in t's binade.
struct SegParams {
    double w;       // sg * 2^(fb - e): q * w is q in units of u, sign-folded
    double us;      // sg * 2^(e - fb): t = us * M
    double rlo, rhi; // |q * w| in [rlo, rhi): the addend is 25..30 binades below the binade
    int32_t lo, hi;  // 2^fb, 2^(fb+1)
    int32_t M0;
};

PG_HD int32_t seg_sat(int32_t v) { return v > SEG_SAT ? SEG_SAT : (v < -SEG_SAT ? -SEG_SAT : v); }

// g after f
PG_HD SegFn seg_then(SegFn f, SegFn g)
{
    SegFn h;
    h.c0 = seg_sat(f.c0 + ((f.c0 & 1) ? g.c1 : g.c0));
    h.c1 = seg_sat(f.c1 + ((f.c1 & 1) ? g.c0 : g.c1));
    return h;
}

PG_HD double seg_pow2(int32_t x, uint32_t neg)
{
    return f64_from_bits(((uint64_t)neg << 63) | ((uint64_t)(uint32_t)(x + 1023) << 52));
}

// false when t is zero or its binade is outside the fast window (no scan then).
PG_HD bool seg_begin(double t, SegParams &sp)
{
    const uint64_t b = f64_bits(t);
    const int32_t e = (int32_t)((b >> 52) & 0x7FF) - 1023;
    if (t == 0.0 || e < FAST_LO || e > FAST_HI)
        return false;
    const uint32_t neg = (uint32_t)(b >> 63);
    const int32_t k = e >> 2;
    const int32_t fb = 28 - ((k ^ (k >> 31)) + 1);
    sp.w = seg_pow2(fb - e, neg);
    sp.us = seg_pow2(e - fb, neg);
    sp.rlo = seg_pow2(fb - 30, 0);
    sp.rhi = seg_pow2(fb - 24, 0);
    sp.lo = 1 << fb;
    sp.hi = 2 << fb;
    sp.M0 = (int32_t)(t * sp.w);
    return true;
}

// The step map of addend q; K and `risky` for the validity test.
PG_HD SegFn seg_fn(double q, const SegParams &sp, int32_t &K, bool &risky)
{
    const double Q = q * sp.w; // exact: a power-of-two scaling of a posit value
    const double aQ = Q < 0 ? -Q : Q;
    risky = (aQ >= sp.rlo) & (aQ < sp.rhi);
    const double Qc = Q > (double)SEG_SAT ? (double)SEG_SAT : (Q < -(double)SEG_SAT ? -(double)SEG_SAT : Q);
    const double Kd = floor(Qc);
    const double F = Qc - Kd; // exact
    K = (int32_t)Kd;
    const int32_t up = F > 0.5, tie = F == 0.5;
    SegFn f;
    f.c0 = K + (up | (tie & (K & 1)));
    f.c1 = K + (up | (tie & ((K + 1) & 1)));
    return f;
}

// Is the step from M exact in the scan form?
PG_HD bool seg_valid(int32_t M, int32_t K, bool risky, const SegParams &sp)
{
    return (M < sp.hi) & (M + K >= sp.lo) & (M + K < sp.hi) & !risky;
}

PG_HD int32_t seg_apply(SegFn f, int32_t M) { return M + ((M & 1) ? f.c1 : f.c0); }

// One step t + q with the exact path behind the FP64 form.
PG_HD double chain_add_one(double t, double q)
{
    uint32_t bad = 0;
    const double r = f64_posit_add(t, q, bad);
    return (bad & 0x40000000u) ? f64_posit_add_exact(t, q) : r;
}



// ---------------------------------------------------------------------------
// The chain step with the fraction width held fixed.
// ---------------------------------------------------------------------------
// In f64_posit_add the rounding constant is built from the sum's exponent with integer
// operations on the dependent path.  Within a range of scales of one fraction width fb the
// posit grid is every number with fb + 1 significant bits, so the rounding is that of the
// FP64 significand to 53 - sh bits (sh = 52 - fb), to nearest, ties to even (the last
// fraction bit is the pattern's), whatever the binade.  Veltkamp's splitting (Dekker, "A
// floating-point technique for extending the available precision", 1971) does exactly
// that in FP64 arithmetic rounded to nearest even: with C = 2^sh + 1, g = fl(C s),
// d = fl(s - g), the high part fl(g + d) is s rounded to 53 - sh bits (2 <= sh <= 51), ties
// to even.  So a step is s = fl(t + q) and three more FP64 operations, no exponent on the
// dependent path.  The fraction width is that of the value a block of steps starts at; it
// is the same in regimes k and -k-1 (both have a run of the same length), so the scales
// [2^-4, 2^4) around 1 form one such range of 8 binades, and the other ranges are single
// regimes.  A step whose sum lands at another fraction width (or is zero, or is risky as in
// f64_posit_add) is flagged, and the caller redoes the block with chain_add_one.
PG_HD int32_t f64_regime(double x) { return ((int32_t)((f64_bits(x) >> 52) & 0x7FF) - 1023) >> 2; }

// The regime run length of the scale of FP64 pattern sb (fb = 28 - run).
PG_HD int32_t f64_bits_run(uint64_t sb)
{
    const int32_t k = ((int32_t)((sb >> 52) & 0x7FF) - 1023) >> 2;
    return (k ^ (k >> 31)) + 1;
}

// C = 2^sh + 1 for regime run `run` (sh = 52 - fb = 24 + run).
PG_HD double f64_split_const(int32_t run) { return f64_add(f64_from_bits((uint64_t)(24 + run + 1023) << 52), 1.0); }

PG_HD double f64_posit_add_split(double t, double q, double C, int32_t run, uint32_t &bad)
{
    const double s = f64_add(t, q);
    const double g = f64_mul(C, s);
    const double r = f64_add(g, f64_add(s, -g));
    // off the dependent path
    const uint64_t sb = f64_bits(s);
    const int32_t et = (int32_t)((f64_bits(t) >> 52) & 0x7FF), eq = (int32_t)((f64_bits(q) >> 52) & 0x7FF);
    const int32_t gap = et > eq ? et - eq : eq - et;
    const bool risky = (eq != 0) & (gap > 24) & (gap <= 30);
    bad |= (risky | (f64_bits_run(sb) != run)) ? 0x40000000u : 0u;
    return r;
}

// t + q_0 + ... + q_{count-1} as chain_add_run, with the fixed-width step: blocks of
// CHAIN_BLOCK steps without a branch, a flagged block redone step by step exactly.
// Terms read from FP64 values or from posit32 patterns (converted on load).
struct TermsF64 {
    const double *q;
    PG_HD_MEMBER double operator[](int i) const { return q[i]; }
    PG_HD_MEMBER TermsF64 operator+(int i) const { return TermsF64{q + i}; }
};
struct TermsP32 {
    const uint32_t *q;
    PG_HD_MEMBER double operator[](int i) const { return p32_to_double(q[i]); }
    PG_HD_MEMBER TermsP32 operator+(int i) const { return TermsP32{q + i}; }
};

template <class Q>
PG_HD double chain_add_run_reg(double t, Q q, int count)
{
    constexpr int U = CHAIN_BLOCK;
    int k = 0;
    for (; k + U <= count; k += U) {
        const int32_t kreg = f64_regime(t);
        const bool in = (t != 0.0) & (kreg >= (FAST_LO >> 2)) & (kreg <= (FAST_HI >> 2));
        const int32_t run = (kreg ^ (kreg >> 31)) + 1;
        const double C = f64_split_const(run);
        double v[U];
#pragma unroll
        for (int j = 0; j < U; ++j)
            v[j] = q[k + j];
        const double t0 = t;
        uint32_t bad = in ? 0u : 0x40000000u;
#pragma unroll
        for (int j = 0; j < U; ++j)
            t = f64_posit_add_split(t, v[j], C, run, bad);
        if (bad & 0x40000000u) { // (from q: a dynamic index into v would put v in local memory)
            t = t0;
            for (int j = 0; j < U; ++j)
                t = chain_add_one(t, q[k + j]);
        }
    }
    for (; k < count; ++k)
        t = chain_add_one(t, q[k]);
    return t;
}

} // namespace pg
