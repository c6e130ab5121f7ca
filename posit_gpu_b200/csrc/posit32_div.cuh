// posit32_div.cuh -- posit32 division and square root with the integer quotient and root
// found from an FP64 estimate.
//
// pdiv and psqrt (posit32.cuh) round the exact quotient / root of the significands: the
// integer quotient q = floor(2^32 g_a / g_b) with its remainder, and the integer root
// r = floor(sqrt(m 2^32)) with its remainder, then pack_exact (the remainder is the sticky
// bit).  Those integers come there from a 64-bit integer division and a bit-by-bit root,
// both long dependent chains.  Here they come from one FP64 division or square root: the
// operands are integers below 2^64 with at most 33 significant bits, so they convert to
// FP64 exactly; the FP64 result is within 2^-20 of the true quotient (below 2^33) or root
// (below 2^32), so its integer part is the true one or one off; the remainder computed in
// 64-bit integer arithmetic (mod 2^64: the true remainder and the one-off ones lie well
// inside the signed range) says which, and one step corrects it.  The integers, and so
// the results, are the same bits as pdiv's and psqrt's.
#pragma once
#include "posit32.cuh"
#include <math.h>

namespace pg {

// floor(num / d) and the remainder, num < 2^63 with at most 33 significant bits,
// 2^30 <= d < 2^31.
PG_HD uint64_t udiv_est(uint64_t num, uint64_t d, uint64_t *rem)
{
    const double qd = (double)num / (double)d;
    uint64_t q = (uint64_t)qd;
    int64_t r = (int64_t)(num - q * d);
    if (r < 0) {
        q -= 1;
        r += (int64_t)d;
    } else if (r >= (int64_t)d) {
        q += 1;
        r -= (int64_t)d;
    }
    *rem = (uint64_t)r;
    return q;
}

// floor(sqrt(x)) and the remainder, x < 2^64 with at most 33 significant bits.
PG_HD uint64_t usqrt_est(uint64_t x, uint64_t *rem)
{
    uint64_t r = (uint64_t)sqrt((double)x);
    int64_t d = (int64_t)(x - r * r); // x - r^2, exact mod 2^64
    if (d < 0) {
        d += (int64_t)(2 * r - 1);    // x - (r-1)^2
        r -= 1;
    } else if (d > (int64_t)(2 * r)) { // x >= (r+1)^2
        d -= (int64_t)(2 * r + 1);
        r += 1;
    }
    *rem = (uint64_t)d;
    return r;
}

// a / b rounded (p32_div; the same bits as pdiv).
PG_HD uint32_t pdiv_est(uint32_t a, uint32_t b)
{
    if (a == P32_NAR || b == P32_NAR || b == 0)
        return P32_NAR;
    if (a == 0)
        return 0;
    const dp32 da = decode(a), db = decode(b);
    uint64_t r;
    const uint64_t q = udiv_est((uint64_t)da.g << 32, db.g, &r);
    const int32_t s = da.s - db.s;
    if (q >> 32)
        return pack_exact(da.x ^ db.x, s, q << 30, r != 0);
    return pack_exact(da.x ^ db.x, s - 1, q << 31, r != 0);
}

// sqrt(a) rounded (the same bits as psqrt).
PG_HD uint32_t psqrt_est(uint32_t a)
{
    if (a == 0)
        return 0;
    if (a >> 31)
        return P32_NAR;
    const dp32 d = decode(a);
    const int32_t odd = d.s & 1;
    const uint64_t m = (uint64_t)d.g << odd;
    uint64_t rem;
    const uint64_t r = usqrt_est(m << 32, &rem);
    return pack_exact(0, (d.s - odd) / 2, r << 31, rem != 0);
}

} // namespace pg
