// posit32.cuh -- posit(32,2) arithmetic for the B200 posit BLAS, compiled for both
// the host and sm_100a.
//
// Bit-exactness target: the SoftPosit algorithm as ported in the reference,
// libRpack/kernel_entry.cl:88-538 (p32_add, p32_mul), including its truncating
// operand alignment and its sticky-bit window, and correctly rounded division and
// square root (no in-tree reference source exists for those two).
//
// Two layers:
//   * pattern-level exact operations (padd, pmul, psub, pdiv, psqrt) -- decode with
//     count-leading-zeros instead of the reference's bit-by-bit regime walk;
//   * the decoded domain used by the GEMM inner loop: a value is held as
//     (scale, significand, sign) with the significand's hidden bit at bit 30, so a
//     multiply-add never re-decodes a bit pattern.  Zero and NaR are encoded as
//     scales far outside the posit range (-1024 and 4096), which makes them fall out
//     of the fast path's range test; the caller then redoes that step exactly.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__ __forceinline__
#define PG_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define PG_HD static inline
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
// Decoded-domain operations for the GEMM inner loop
// ----------------------------------------------------------------------------

// Round a value whose significand T-window has already been formed: `thi` holds the
// hidden bit and the kept fraction bits (hidden at bit 28-run), `tlo` the guard bit
// (bit 31) and the sticky bits (30..0).  Round to nearest even on the last kept bit.
PG_HD void round_window(uint32_t thi, uint32_t tlo, int32_t s, uint32_t run, dp32 &r)
{
    uint32_t up = (tlo | (thi & 1u)) > 0x80000000u ? 1u : 0u;
    uint32_t g = shl32(thi + up, run + 2); // hidden back at bit 30, or 31 on carry-out
    uint32_t ov = g >> 31;
    r.s = s + (int32_t)ov;
    r.g = g >> ov;
}

PG_HD uint32_t regime_run(int32_t s)
{
    int32_t k = s >> 2;
    return (uint32_t)((k ^ (k >> 31)) + 1);
}

PG_HD bool in_fast_range(int32_t s) { return (uint32_t)(s - FAST_LO) <= (uint32_t)(FAST_HI - FAST_LO); }

// t*a rounded to posit32, both operands decoded.  Returns false (result unusable) if
// the result's regime is longer than 27 bits, or an operand is zero or NaR.
PG_HD bool dmul_fast(const dp32 &t, const dp32 &a, dp32 &r)
{
    uint64_t p = (uint64_t)t.g * a.g;
    uint32_t hi = (uint32_t)(p >> 32), lo = (uint32_t)p;
    uint32_t carry = hi >> 29; // hidden bit at 61 instead of 60
    int32_t s = t.s + a.s + (int32_t)carry;
    uint32_t run = regime_run(s);
    uint32_t sh = run + carry; // the reference's (frac >> carry) >> run
    uint32_t tlo = shr64_lo(lo, hi, sh);
    uint32_t thi = shr32(hi, sh);
    round_window(thi, tlo, s, run, r);
    r.x = t.x ^ a.x;
    return in_fast_range(s);
}

// c + p rounded to posit32, both decoded.  Returns false if the exact path is needed:
// result regime longer than 27 bits, NaR, or an exactly zero sum.
PG_HD bool dadd_fast(const dp32 &c, const dp32 &p, dp32 &r)
{
    int32_t d = c.s - p.s;
    bool sw = d < 0;
    int32_t bs = sw ? p.s : c.s;
    uint32_t bg = sw ? p.g : c.g;
    uint32_t bx = sw ? p.x : c.x;
    uint32_t sg = sw ? c.g : p.g;
    uint32_t ad = (uint32_t)(sw ? -d : d);
    ad = ad > 63u ? 63u : ad;
    // the smaller operand in the 64-bit frame (hidden at 62), truncated at bit 0
    uint64_t B = ((uint64_t)sg << 32) >> ad;
    uint64_t A = (uint64_t)bg << 32;
    uint64_t S = (c.x ^ p.x) ? A - B : A + B;
    // equal scales and opposite signs may leave a negative difference
    uint32_t neg = (uint32_t)(S >> 63) & (c.x ^ p.x);
    S = neg ? 0ull - S : S;
    uint32_t shi = (uint32_t)(S >> 32);
    uint32_t lz = clz32(shi); // S.hi == 0 only when S == 0
    // normalise to the hidden bit at 63 (bits shifted in are zero); lz <= 32
    uint64_t N = S << lz;
    uint32_t nhi = (uint32_t)(N >> 32), nlo = (uint32_t)N;
    int32_t s = bs + 1 - (int32_t)lz;
    uint32_t run = regime_run(s);
    uint32_t sh = run + 3;
    uint32_t tlo = shr64_lo(nlo, nhi, sh);
    uint32_t thi = shr32(nhi, sh);
    round_window(thi, tlo, s, run, r);
    r.x = bx ^ neg;
    return in_fast_range(s) && shi != 0;
}

// Exact decoded operations (through patterns): the slow path.
PG_HD_NOINLINE dp32 dmul_exact(dp32 t, dp32 a) { return decode(pmul(encode(t), encode(a))); }
PG_HD_NOINLINE dp32 dadd_exact(dp32 c, dp32 p) { return decode(padd(encode(c), encode(p))); }
PG_HD_NOINLINE dp32 dmac_exact(dp32 c, dp32 t, dp32 a)
{
    return decode(padd(encode(c), pmul(encode(t), encode(a))));
}

// c + t*a with both roundings; never fails.
PG_HD dp32 dmac(const dp32 &c, const dp32 &t, const dp32 &a)
{
    dp32 p, r;
    bool ok = dmul_fast(t, a, p);
    ok = dadd_fast(c, p, r) && ok;
    if (!ok)
        r = dmac_exact(c, t, a);
    return r;
}

} // namespace pg
