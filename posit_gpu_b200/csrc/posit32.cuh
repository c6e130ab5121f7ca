// posit32.cuh -- posit(32,2) arithmetic for the B200 posit BLAS, compiled for both
// the host and sm_100a.
//
// Bit-exactness target: the SoftPosit algorithm as ported in the reference,
// libRpack/kernel_entry.cl:88-538 (p32_add, p32_mul), including its truncating
// operand alignment and its sticky-bit window, and correctly rounded division and
// square root (no in-tree reference source exists for those two).
//
// Three layers:
//   * pattern-level exact operations (padd, pmul, psub, pdiv, psqrt) -- decode with
//     count-leading-zeros instead of the reference's bit-by-bit regime walk; the exact
//     path of the two fast forms below;
//   * the FP64 form (end of this file): posit values held in FP64, one multiply-add as a
//     few FP64 operations that round onto the posit grid -- the GEMM, the column
//     solves and the batched factorizations;
//   * the decoded integer form: a value held as (scale, significand, sign) with the
//     significand's hidden bit at bit 30 -- the one-thread triangular-solve chain
//     (trsm_chain.cuh).  Zero is a scale far below the posit range, NaR stays outside
//     (the callers carry it as a flag).
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__ __forceinline__
#define PG_HD_MEMBER __host__ __device__ __forceinline__
#define PG_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define PG_HD static inline
#define PG_HD_MEMBER inline
#define PG_HD_NOINLINE static
#endif

namespace pg {

constexpr uint32_t P32_NAR = 0x80000000u;
constexpr uint32_t P32_ONE = 0x40000000u;
constexpr uint32_t P32_MAXPOS = 0x7FFFFFFFu;
constexpr int32_t ZERO_SCALE = -1024;
constexpr int32_t NAR_SCALE = 4096;
// The fast paths below are exact whenever the result scale lies in this window,
// i.e. whenever the result's regime run is at most 27 bits long.
constexpr int32_t FAST_LO = -108;
constexpr int32_t FAST_HI = 107;

PG_HD uint32_t clz32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__clz((int)x);
#else
    return x ? (uint32_t)__builtin_clz(x) : 32u;
#endif
}

// (hi:lo) >> n for 0 <= n <= 32, low word.
PG_HD uint32_t shr64_lo(uint32_t lo, uint32_t hi, uint32_t n)
{
#if defined(__CUDA_ARCH__)
    return __funnelshift_rc(lo, hi, n);
#else
    return n >= 32 ? hi : (uint32_t)((((uint64_t)hi << 32) | lo) >> n);
#endif
}

// Shifts with amounts clamped to 32 (defined for any n; one funnel shift on the GPU).
PG_HD uint32_t shr32(uint32_t x, uint32_t n)
{
#if defined(__CUDA_ARCH__)
    return __funnelshift_rc(x, 0u, n);
#else
    return n >= 32 ? 0u : x >> n;
#endif
}
PG_HD uint32_t shl32(uint32_t x, uint32_t n)
{
#if defined(__CUDA_ARCH__)
    return __funnelshift_lc(0u, x, n);
#else
    return n >= 32 ? 0u : x << n;
#endif
}

// ----------------------------------------------------------------------------
// Decoded representation
// ----------------------------------------------------------------------------
struct dp32 {
    int32_t s;  // scale: value = (-1)^x * 2^s * g / 2^30
    uint32_t g; // significand, hidden bit at 30 (0 for zero)
    uint32_t x; // sign, 0 or 1
};

// Pattern -> decoded.  Regime run length by count-leading-zeros (the reference walks
// it bit by bit, kernel_entry.cl:112-130).
PG_HD dp32 decode(uint32_t u)
{
    dp32 r;
    if (u == 0) {
        r.s = ZERO_SCALE;
        r.g = 0;
        r.x = 0;
        return r;
    }
    if (u == P32_NAR) {
        r.s = NAR_SCALE;
        r.g = P32_ONE;
        r.x = 0;
        return r;
    }
    r.x = u >> 31;
    uint32_t v = r.x ? 0u - u : u;
    uint32_t y = v << 1;
    uint32_t ones = v & 0x40000000u;
    uint32_t run = ones ? clz32(~y) : clz32(y);
    int32_t k = ones ? (int32_t)run - 1 : -(int32_t)run;
    uint32_t rest = shl32(v, run + 2); // exponent at 31..30, fraction below
    r.s = 4 * k + (int32_t)(rest >> 30);
    r.g = P32_ONE | (rest & 0x3FFFFFFFu);
    return r;
}

// Pack with the reference's rounding (kernel_entry.cl:167-216): the significand has
// its hidden bit at bit 62; the part below is shifted right by run+2, bits falling off
// the 64-bit word are lost, bit 31 of the shifted word is the guard bit and bits 30..0
// are the sticky bits (for every run length); |k| > 30 saturates.
PG_HD uint32_t pack_sp(uint32_t neg, int32_t scale, uint64_t sig62)
{
    int32_t k = scale >> 2;
    int32_t e = scale & 3;
    int32_t run = (k < 0) ? -k : k + 1;
    uint32_t u;
    if (run > 30) {
        u = (k < 0) ? 1u : P32_MAXPOS;
    } else {
        uint32_t regime = (k < 0) ? (0x40000000u >> run) : (0x7FFFFFFFu ^ (0x7FFFFFFFu >> run));
        uint64_t tail = (sig62 & 0x3FFFFFFFFFFFFFFFull) >> (run + 2);
        uint32_t ebits, guard;
        if (run <= 28) {
            ebits = (uint32_t)e << (28 - run);
            guard = (uint32_t)(tail >> 31) & 1u;
        } else if (run == 29) {
            ebits = (uint32_t)e >> 1;
            guard = (uint32_t)e & 1u;
        } else {
            ebits = 0;
            guard = ((uint32_t)e >> 1) & 1u;
        }
        u = regime + ebits + (uint32_t)(tail >> 32);
        if (guard)
            u += (u & 1u) | (uint32_t)((tail & 0x7FFFFFFFull) != 0);
    }
    return neg ? 0u - u : u;
}

// Decoded -> pattern.  Exact for every value produced by this file's operations.
PG_HD uint32_t encode(const dp32 &d)
{
    if (d.s >= 2048)
        return P32_NAR;
    if (d.g == 0 || d.s <= -512)
        return 0u;
    return pack_sp(d.x, d.s, (uint64_t)d.g << 32);
}

// ----------------------------------------------------------------------------
// Exact operations on patterns
// ----------------------------------------------------------------------------

// kernel_entry.cl:399-538.  NaR first, then zero.
PG_HD uint32_t pmul(uint32_t a, uint32_t b)
{
    if (a == P32_NAR || b == P32_NAR)
        return P32_NAR;
    if (a == 0 || b == 0)
        return 0;
    dp32 da = decode(a), db = decode(b);
    uint64_t p = (uint64_t)da.g * db.g; // hidden bit at 60 or 61
    int32_t s = da.s + db.s;
    if (p >> 61) {
        s += 1;
        p >>= 1;
    }
    return pack_sp(da.x ^ db.x, s, p << 2);
}

// kernel_entry.cl:370-397 with addMags (88-217) and subMags (219-368).
PG_HD uint32_t padd(uint32_t a, uint32_t b)
{
    if (a == 0 || b == 0)
        return a | b;
    if (a == P32_NAR || b == P32_NAR)
        return P32_NAR;
    uint32_t ma = (a >> 31) ? 0u - a : a;
    uint32_t mb = (b >> 31) ? 0u - b : b;
    bool diff = ((a ^ b) >> 31) != 0;
    if (diff && ma == mb)
        return 0;
    // order by magnitude; the larger operand's sign is the result's
    uint32_t big = a, small = b;
    if (mb > ma) {
        big = b;
        small = a;
    }
    dp32 db = decode(big), ds = decode(small);
    uint64_t A = (uint64_t)db.g << 32, B = (uint64_t)ds.g << 32;
    int32_t shift = db.s - ds.s;
    int32_t s = db.s;
    if (!diff) {
        A += (shift > 63) ? 0 : (B >> shift);
        if (A >> 63) {
            s += 1;
            A >>= 1;
        }
    } else {
        if (shift > 63)
            return big;
        A -= B >> shift;
        while (!(A >> 62)) {
            A <<= 1;
            s -= 1;
        }
    }
    return pack_sp(db.x, s, A);
}

PG_HD uint32_t psub(uint32_t a, uint32_t b) { return padd(a, 0u - b); }

// Correctly rounded packing (posit standard: nearest, ties to the even pattern, never
// to zero or NaR) of 2^scale * sig/2^62 plus `sticky` below sig's last bit.
PG_HD uint32_t pack_exact(uint32_t neg, int32_t scale, uint64_t sig62, uint32_t sticky)
{
    int32_t k = scale >> 2, e = scale & 3;
    uint32_t u;
    if (k >= 30) {
        u = P32_MAXPOS;
    } else if (k < -30) {
        u = 1u;
    } else {
        int32_t run = (k < 0) ? -k : k + 1;
        // 31-bit body: regime+terminator (run+1), exponent (2), fraction (28-run).
        // Build it in a 64-bit word left-aligned at bit 63, fraction bits following.
        uint64_t frac = sig62 & 0x3FFFFFFFFFFFFFFFull; // 62 fraction bits
        uint64_t w;                                    // body bits from bit 63 down
        uint32_t extra_sticky = 0;
        uint64_t head = (k < 0) ? 1ull : ((((uint64_t)1 << run) - 1) << 1); // run+1 bits
        int32_t hb = run + 1 + 2;                                               // head+exp bits
        w = ((head << 2) | (uint64_t)e) << (64 - hb);
        // append fraction below the exponent: bits (63-hb) .. 0 hold frac's top bits
        w |= frac >> (hb - 2);
        extra_sticky = (frac & ((((uint64_t)1) << (hb - 2)) - 1)) != 0;
        // w holds at least 33 significant body bits: keep 31, round on the rest
        uint32_t body = (uint32_t)(w >> 33);
        uint64_t rem = w & 0x1FFFFFFFFull;
        uint64_t half = 0x100000000ull;
        uint32_t st = sticky | extra_sticky;
        if (rem > half || (rem == half && (st || (body & 1u))))
            body += 1;
        u = body;
    }
    return neg ? 0u - u : u;
}

PG_HD uint32_t pdiv(uint32_t a, uint32_t b)
{
    if (a == P32_NAR || b == P32_NAR || b == 0)
        return P32_NAR;
    if (a == 0)
        return 0;
    dp32 da = decode(a), db = decode(b);
    uint64_t num = (uint64_t)da.g << 32;
    uint64_t q = num / db.g, r = num % db.g;
    int32_t s = da.s - db.s;
    if (q >> 32)
        return pack_exact(da.x ^ db.x, s, q << 30, r != 0);
    return pack_exact(da.x ^ db.x, s - 1, q << 31, r != 0);
}

PG_HD uint64_t isqrt64(uint64_t x, uint64_t *rem)
{
    uint64_t res = 0, bit = (uint64_t)1 << 62;
    while (bit > x)
        bit >>= 2;
    while (bit) {
        if (x >= res + bit) {
            x -= res + bit;
            res = (res >> 1) + bit;
        } else {
            res >>= 1;
        }
        bit >>= 2;
    }
    *rem = x;
    return res;
}

PG_HD uint32_t psqrt(uint32_t a)
{
    if (a == 0)
        return 0;
    if (a >> 31)
        return P32_NAR;
    dp32 d = decode(a);
    int32_t odd = d.s & 1;
    uint64_t m = (uint64_t)d.g << odd;
    uint64_t rem;
    uint64_t r = isqrt64(m << 32, &rem);
    return pack_exact(0, (d.s - odd) / 2, r << 31, rem != 0);
}

// IEEE double -> posit32, correctly rounded (nearest, ties to even pattern; never to
// zero or NaR).  SoftPosit's convertDoubleToP32 has no in-tree source: unpinned.
PG_HD uint32_t p32_from_double(double x)
{
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    uint32_t neg = (uint32_t)(b >> 63);
    int32_t ex = (int32_t)((b >> 52) & 0x7FF);
    uint64_t man = b & 0xFFFFFFFFFFFFFull;
    if (ex == 0x7FF)
        return P32_NAR; // inf / nan
    if (ex == 0) {
        if (man == 0)
            return 0;
        return neg ? 0u - 1u : 1u; // subnormal doubles lie far below minpos
    }
    uint64_t sig62 = ((uint64_t)1 << 62) | (man << 10);
    return pack_exact(neg, ex - 1023, sig62, 0);
}

// posit32 -> IEEE double (exact).  NaR -> quiet NaN.
PG_HD double p32_to_double(uint32_t u)
{
    uint64_t b;
    if (u == 0) {
        b = 0;
    } else if (u == P32_NAR) {
        b = 0x7FF8000000000000ull;
    } else {
        dp32 d = decode(u);
        uint64_t man = ((uint64_t)(d.g & 0x3FFFFFFFu)) << 22; // 30 fraction bits -> 52
        b = ((uint64_t)d.x << 63) | ((uint64_t)(d.s + 1023) << 52) | man;
    }
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
}

PG_HD uint32_t pneg(uint32_t a) { return 0u - a; }
PG_HD uint32_t pabs(uint32_t a) { return ((int32_t)a < 0) ? 0u - a : a; }

// ----------------------------------------------------------------------------
// Decoded integer form (the one-thread chain of trsm_chain.cuh)
// ----------------------------------------------------------------------------
//
// Integer code written to put as much of its work as possible on the integer
// multiply-add pipe:
//   * every quantity that depends only on a result's scale (regime run length, the
//     multipliers that shift by it, whether the fast path is exact there) comes from
//     regime_entry, computed from that scale;
//   * right shifts by n are multiplies by 2^(32-n) keeping the high word, and a 64-bit
//     funnel shift is two multiply-adds;
//   * round-to-nearest-even at bit 32 is one 64-bit add of 0x7FFFFFFF + lsb.
// In the fast path the smaller addend is shifted by at most 30 bits inside a 64-bit
// frame, so no bit of it is lost and the sum is exact: the reference's truncating
// alignment (kernel_entry.cl:154, 292-298) can only matter beyond that, where the step
// is handed to the exact path instead.

// Multiply-high and 64-bit multiply-add (single integer multiply-add instructions).
PG_HD uint32_t umulhi(uint32_t a, uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// Round to nearest even at bit 32 of (thi:tlo), returning the rounded high word:
// thi + carry-out of (tlo | lsb) + 0x7FFFFFFF.  On the GPU this is one 32x32+64-bit
// multiply-add (integer multiply-add pipe) instead of an add-with-carry pair.
PG_HD uint32_t round_hi(uint32_t thi, uint32_t tlo)
{
    uint32_t v = tlo | (thi & 1u);
#if defined(__CUDA_ARCH__)
    uint64_t acc = ((uint64_t)thi << 32) | 0x7FFFFFFFu, r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(v), "r"(1u), "l"(acc));
    return (uint32_t)(r >> 32);
#else
    return thi + (uint32_t)(((uint64_t)v + 0x7FFFFFFFu) >> 32);
#endif
}

PG_HD uint32_t regime_run(int32_t s)
{
    int32_t k = s >> 2;
    return (uint32_t)((k ^ (k >> 31)) + 1);
}

PG_HD bool in_fast_range(int32_t s) { return (uint32_t)(s - FAST_LO) <= (uint32_t)(FAST_HI - FAST_LO); }

// Decoded zero.  Any product with a zero operand then has a
// scale <= DECODED_ZERO_SCALE + 121 < ZERO_REGION, below every nonzero product (>= -241) and
// every nonzero sum (>= -270), and its significand is 0.
constexpr int32_t DECODED_ZERO_SCALE = -512;
constexpr int32_t ZERO_REGION = -300;

// Per result scale s: the rounding parameters of the decoded integer form (regime_entry).
struct RegimeEntry {
    uint32_t r0;  // 2^(32-run): umulhi by it shifts right by run
    uint32_t nr1; // -(2^(31-run)); r0 + carry*nr1 = 2^(32-run-carry).  Bit 30 set
                  // means "a zero significand here is a failure" (clear in the zero region)
    uint32_t g;   // 2^(run+2): moves the kept bits back to a hidden bit at 30
    uint32_t w;   // 2^(29-run) (window multiplier for a hidden bit at 63), bit 30 = fail
};

PG_HD RegimeEntry regime_entry(int32_t s)
{
    RegimeEntry e;
    // bitwise, not short-circuit, operators: this also runs on a dependent path, where a
    // branch would stop independent work from overlapping it
    const bool zero_region = s < ZERO_REGION;
    const bool fast = in_fast_range(s); // the fast window lies above the zero region
    const uint32_t run = fast ? regime_run(s) : 27u;
    e.r0 = 1u << (32 - run);
    e.nr1 = zero_region ? 0u : 0u - (1u << (31 - run));
    e.g = 1u << (run + 2);
    e.w = (1u << (29 - run)) | ((fast | zero_region) ? 0u : 0x40000000u);
    return e;
}

// Regime entry by arithmetic: one thread's chain of dependent additions, where a table
// load would sit on the dependent path.
struct ComputedEntry {
    PG_HD_MEMBER RegimeEntry operator()(int32_t s) const { return regime_entry(s); }
};

// t*a rounded to posit32 (kernel_entry.cl:399-538), both operands decoded and nonzero
// or decoded zeros.  `bad` gets bit 30 set when the result must come from the exact path
// (regime longer than 27 bits, or rounding carried out of the significand).
template <class EntryOf>
PG_HD void dmul_core(const dp32 &t, const dp32 &a, EntryOf entry_of, dp32 &r, uint32_t &bad)
{
    uint64_t P = (uint64_t)t.g * a.g; // hidden bit at 60, or 61 ("carry")
    uint32_t hi = (uint32_t)(P >> 32), lo = (uint32_t)P;
    uint32_t carry = umulhi(hi, 8u);
    int32_t s = t.s + a.s + (int32_t)carry;
    const RegimeEntry e = entry_of(s);
    uint32_t W = e.r0 + carry * e.nr1; // 2^(32 - run - carry)
    // T = P >> (run + carry): kept bits in thi (hidden at 28-run), guard+sticky in tlo
    uint32_t thi = umulhi(hi, W);
    uint32_t tlo = hi * W + umulhi(lo, W);
    r.g = round_hi(thi, tlo) * e.g;
    r.s = s;
    r.x = t.x ^ a.x;
    bad = e.w | (~r.g & e.nr1);
}

// c + p rounded to posit32 (kernel_entry.cl:370-397), both decoded.  Fails (bit 30 of
// `bad`) for a result regime longer than 27 bits, an exactly cancelling sum of nonzero
// values, or a rounding carry-out.
// An addend more than 30 binades below the other contributes nothing here (Q = 0), and
// that is also the reference's result: in its 64-bit frame (hidden bit at 62) such an
// addend is below 2^32, i.e. entirely under the guard bit of the larger operand, whose
// bits below its last kept bit are zero.  A sum then rounds back to the larger operand;
// a difference A - e (0 < e < 2^32) borrows ones through every bit up to A's last kept
// bit, so guard and sticky are set and it rounds up to A again -- including when A is a
// power of two, since the spacing below A is at least 2^(33+run) frame units.
template <class EntryOf>
PG_HD void dadd_core(const dp32 &c, const dp32 &p, EntryOf entry_of, dp32 &r, uint32_t &bad)
{
    // order by magnitude: scale, then significand (so the difference is never negative).
    // Bitwise, not short-circuit, operators: the latter compile to branches, which both
    // cost issue slots and stop the scheduler from interleaving independent steps.
    bool sw = (c.s < p.s) | ((c.s == p.s) & (c.g < p.g));
    int32_t bs = sw ? p.s : c.s;
    uint32_t bg = sw ? p.g : c.g;
    uint32_t sg = sw ? c.g : p.g;
    uint32_t bx = sw ? p.x : c.x;
    int32_t d = c.s - p.s;
    uint32_t ad = (uint32_t)(d < 0 ? -d : d);
    uint32_t Q = shr32(0x40000000u, ad); // 2^(30-ad); 0 beyond 30
    int32_t M = (c.x ^ p.x) ? -(int32_t)Q : (int32_t)Q;
    // frame: the larger significand's hidden bit at 60; exact for ad <= 30
    uint64_t S = (uint64_t)(((int64_t)bg << 30) + (int64_t)(int32_t)sg * (int64_t)M);
    uint32_t shi = (uint32_t)(S >> 32), slo = (uint32_t)S;
    uint32_t lz = clz32(shi);         // S.hi == 0 only when S == 0
    int32_t s = bs + 3 - (int32_t)lz; // result scale
    const RegimeEntry e = entry_of(s);
    uint32_t p2 = shl32(1u, lz);
    uint32_t nhi = shi * p2 + umulhi(slo, p2); // N = S << lz: hidden bit at 63
    uint32_t nlo = slo * p2;
    uint32_t thi = umulhi(nhi, e.w); // T = N >> (run + 3)
    uint32_t tlo = nhi * e.w + umulhi(nlo, e.w);
    r.g = round_hi(thi, tlo) * e.g;
    r.s = s;
    r.x = bx;
    bad = e.w | (~r.g & e.nr1);
}

// Exact decoded operations (through patterns): the slow path.  Decoded zeros
// (significand 0) encode to the zero pattern.
PG_HD_NOINLINE dp32 dmac_exact(dp32 c, dp32 t, dp32 a)
{
    dp32 r = decode(padd(encode(c), pmul(encode(t), encode(a))));
    if (r.g == 0)
        r.s = DECODED_ZERO_SCALE;
    return r;
}

// Decode with zero at DECODED_ZERO_SCALE; NaR is the caller's business.
PG_HD dp32 decode_dz(uint32_t u)
{
    dp32 d = decode(u);
    if (u == 0)
        d.s = DECODED_ZERO_SCALE;
    return d;
}

// decode_dz without branches (selects only), for a thread's dependent chain, where a
// branch would stop the next step's independent work from overlapping the current one.
// u must not be NaR.
PG_HD dp32 decode_dz_bf(uint32_t u)
{
    const uint32_t x = u >> 31;
    const uint32_t v = x ? 0u - u : u;
    const uint32_t y = v << 1;
    const uint32_t ones = v & 0x40000000u;
    const uint32_t run = clz32(ones ? ~y : y);
    const int32_t k = ones ? (int32_t)run - 1 : -(int32_t)run;
    const uint32_t rest = shl32(v, run + 2); // exponent at 31..30, fraction below
    dp32 r;
    r.s = u == 0 ? DECODED_ZERO_SCALE : 4 * k + (int32_t)(rest >> 30);
    r.g = u == 0 ? 0u : (P32_ONE | (rest & 0x3FFFFFFFu));
    r.x = x;
    return r;
}

// c + t*a with both roundings, for one thread's chain of dependent multiply-adds (the
// dot-form triangular solve, Rtrsm.cpp:175-186, as c - l*b = c + (-b)*l).  Only the
// addition depends on the previous step; the product, the operands' decoding and the
// exactness test are independent of it and overlap the chain.  Regime entries are
// computed (no table load on the dependent path); flagged steps go through the exact
// routines.  Never fails.
PG_HD dp32 dmac_chain(const dp32 &c, const dp32 &t, const dp32 &a)
{
    dp32 p, r;
    uint32_t bm, ba;
    dmul_core(t, a, ComputedEntry{}, p, bm);
    dadd_core(c, p, ComputedEntry{}, r, ba);
    if ((bm | ba) & 0x40000000u)
        r = dmac_exact(c, t, a);
    return r;
}

// ----------------------------------------------------------------------------
// FP64 form
// ----------------------------------------------------------------------------
// A posit32 value is exact in FP64 (at most 28 significant bits, scale within +-120), so
// p32_mul and p32_add can run on FP64 values: an FP64 operation, then rounding to the
// posit's fraction width at the result's binade -- round to nearest even at the posit's
// last fraction bit, done by adding and subtracting C = 1.5 * 2^(e + 52 - fb) (e the
// binade, fb = 28 - regime run the fraction width).  The even pattern of posit rounding is
// the even fraction, so this is the posit rounding wherever fb >= 1 (the fast window).
PG_HD uint64_t f64_bits(double x)
{
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
}
PG_HD double f64_from_bits(uint64_t b)
{
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
}
PG_HD double f64_add(double a, double b)
{
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b); // never contracted or reassociated
#else
    return a + b;
#endif
}

// C = 1.5 * 2^(e + 52 - fb) for the binade (biased FP64 exponent field) `eb`, as the
// high word of a double whose low word is 0.
PG_HD uint32_t f64_round_const_hi(int32_t eb)
{
    const int32_t k = (eb - 1023) >> 2;     // regime value
    const int32_t run = (k ^ (k >> 31)) + 1; // regime run; fb = 28 - run
    return ((uint32_t)(eb + 24 + run) << 20) | 0x00080000u;
}

PG_HD double f64_fma(double a, double b, double c)
{
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}
PG_HD double f64_mul(double a, double b)
{
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

PG_HD bool f64_outside_fast(int32_t eb)
{
    return (uint32_t)(eb - 1023 - FAST_LO) > (uint32_t)(FAST_HI - FAST_LO);
}

// Biased FP64 exponent field (the binade) of x.
PG_HD int32_t f64_binade(double x) { return (int32_t)((f64_bits(x) >> 52) & 0x7FF); }

// High and low 32-bit words of an FP64 value, and an FP64 value from its high word (low
// word 0: every rounding constant is one).
PG_HD uint32_t f64_hi(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__double2hiint(x);
#else
    return (uint32_t)(f64_bits(x) >> 32);
#endif
}
PG_HD double f64_from_hi(uint32_t h)
{
#if defined(__CUDA_ARCH__)
    return __hiloint2double((int)h, 0);
#else
    return f64_from_bits((uint64_t)h << 32);
#endif
}

// The rounding constant's high word for an FP64 value whose top 12 bits (sign and
// exponent field) are `top`: C = 1.5 * 2^(e + 52 - fb), the same for either sign.  A binade
// outside the fast window gets a NaN instead, so that a product or sum falling there comes
// out NaN and is redone exactly.  Binade 0 holds zero (a zero product or an exactly
// cancelling sum): in the window.
PG_HD uint32_t f64_round_const_top(uint32_t top)
{
    const int32_t eb = (int32_t)(top & 0x7FF);
    if (eb != 0 && f64_outside_fast(eb))
        return 0x7FF80000u;
    return f64_round_const_hi(eb);
}
// The table the GEMM kernels keep in shared memory: f64_round_const_top for every top
// 12 bits, so that a lookup is one shift of the value's high word.
constexpr int F64_CONST_ENTRIES = 4096;
struct F64ConstTable {
    const uint32_t *tab;
    PG_HD_MEMBER uint32_t hi(double x) const { return tab[f64_hi(x) >> 20]; }
    PG_HD_MEMBER double operator()(double x) const { return f64_from_hi(hi(x)); }
};
struct F64ConstTable8 {
    const double *tab;
    PG_HD_MEMBER uint32_t hi(double x) const { return f64_hi(tab[f64_hi(x) >> 20]); }
    PG_HD_MEMBER double operator()(double x) const { return tab[f64_hi(x) >> 20]; }
};
struct F64ConstComputed {
    PG_HD_MEMBER uint32_t hi(double x) const { return f64_round_const_top(f64_hi(x) >> 20); }
    PG_HD_MEMBER double operator()(double x) const { return f64_from_hi(hi(x)); }
};

// c + t*a with both roundings (p32_mul, kernel_entry.cl:399-538, then p32_add,
// kernel_entry.cl:370-397), all three posit32 values held in FP64:
//   q = fma(t, a, Cp) - Cp    the exact product rounded once to the posit grid of its
//                             binade (taken from fl(t*a); where that rounds up to a power
//                             of two both give that power);
//   s = c + q                 the FP64 sum, tested for exactness: s - c == q and s - q == c
//                             (Fast2Sum on the larger operand makes an inexact s fail it);
//   r = (s + Cs) - Cs         the exact sum rounded to the posit grid of its binade.
// `fail` is set when the step must be done exactly instead: an inexact FP64 sum (a
// product outside the fast window has a NaN constant, so q and s are NaN and fail the
// test), or a sum outside the fast window (its table entry is the NaN marker).
// Flagging every inexact sum is conservative: beyond 30 binades the rounded sum would be
// right anyway, but that case is rare on the data the GEMM sees.
template <class ConstOf>
PG_HD double f64_posit_mac(double c, double t, double a, ConstOf const_of, bool &fail)
{
    const double p = f64_mul(t, a);
    const double Cp = const_of(p);
    const double q = f64_add(f64_fma(t, a, Cp), -Cp);
    const double s = f64_add(c, q);
    // s is exact iff s - c == q and s - q == c: with the operands ordered by exponent,
    // s - larger is exact (Dekker's Fast2Sum), so an inexact s leaves that difference
    // unequal to the smaller operand
    const bool inexact = (f64_add(s, -c) != q) | (f64_add(s, -q) != c);
    const uint32_t cs_hi = const_of.hi(s);
    const double Cs = f64_from_hi(cs_hi);
    const double r = f64_add(f64_add(s, Cs), -Cs);
    fail = inexact | (cs_hi == 0x7FF80000u); // the sum's binade is outside the fast window
    return r;
}

// The same step on patterns (the exact path).  Inlined: a called function in the GEMM
// kernels' inner loop made them fault and crawl on inputs that take this path often.
PG_HD double f64_posit_mac_exact(double c, double t, double a)
{
    return p32_to_double(padd(p32_from_double(c), pmul(p32_from_double(t), p32_from_double(a))));
}

// c + t*a with the exact path taken where the FP64 step is flagged.
PG_HD double f64_posit_mac_checked(double c, double t, double a)
{
    bool fail;
    const double r = f64_posit_mac(c, t, a, F64ConstComputed{}, fail);
    return fail ? f64_posit_mac_exact(c, t, a) : r;
}

// The same with the constants from a table.
template <class ConstOf>
PG_HD double f64_posit_mac_checked(double c, double t, double a, ConstOf const_of)
{
    bool fail;
    const double r = f64_posit_mac(c, t, a, const_of, fail);
    return fail ? f64_posit_mac_exact(c, t, a) : r;
}

// x*y rounded as p32_mul (kernel_entry.cl:399-538) rounds it, both posit32 values held in
// FP64: the exact product rounded once onto the posit grid of its binade, fma(x, y, Cp) - Cp
// (the product step of f64_posit_mac).  A product outside the fast window (its constant is
// NaN) and NaR operands (NaN) go through the pattern routine.
template <class ConstOf>
PG_HD double f64_posit_mul_checked(double x, double y, ConstOf const_of)
{
    const double Cp = const_of(f64_mul(x, y));
    const double q = f64_add(f64_fma(x, y, Cp), -Cp);
    return q == q ? q : p32_to_double(pmul(p32_from_double(x), p32_from_double(y)));
}

// FP64 -> posit32 for a value that IS a posit32 value (an output of the FP64 steps or of
// p32_to_double): the fields are assembled without rounding.  Regimes longer than 27 bits
// (fewer than one fraction bit) and NaN go through p32_from_double.
PG_HD uint32_t p32_from_double_exact(double x)
{
    const uint64_t b = f64_bits(x);
    const int32_t s = (int32_t)((b >> 52) & 0x7FF) - 1023;
    if ((b << 1) == 0)
        return 0;
    if ((uint32_t)(s - FAST_LO) > (uint32_t)(FAST_HI - FAST_LO))
        return p32_from_double(x);
    const int32_t k = s >> 2;
    const uint32_t run = (uint32_t)((k ^ (k >> 31)) + 1); // regime run; fraction bits 28 - run
    const uint32_t reg = k >= 0 ? ((1u << run) - 1u) << 1 : 1u; // the run+1 regime bits
    const uint32_t u = (reg << (30 - run)) | ((uint32_t)(s & 3) << (28 - run)) |
                       (uint32_t)((b & 0xFFFFFFFFFFFFFull) >> (24 + run));
    return (b >> 63) ? 0u - u : u;
}

} // namespace pg
