/*
 * posit_oracle.c -- CPU restatement of the reference posit(32,2) arithmetic and of
 * the posit BLAS/LAPACK operation orders (test infrastructure; see posit_oracle.h).
 *
 * Every routine follows the reference step by step where the bits depend on it
 * (operation order, truncation, rounding window); the code itself is written for
 * this project.  Each function names the reference lines it restates.
 */
#include "posit_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NAR ORC_P32_NAR
#define ONE ORC_P32_ONE

/* ------------------------------------------------------------------------- */
/* Arithmetic                                                                */
/* ------------------------------------------------------------------------- */

/* Regime / exponent / fraction of a positive, nonzero, non-NaR pattern, walking the
 * regime run one bit at a time (kernel_entry.cl:109-130 and 434-452).
 * f receives the significand with its hidden bit at bit 30. */
static void orc_fields(uint32_t u, int *k, int *e, uint32_t *f)
{
    uint32_t w = u << 2; /* sign bit and first regime bit shifted out */
    int kk;
    if (u & 0x40000000u) {
        kk = 0;
        while (w & 0x80000000u) { /* further ones of the run */
            kk++;
            w <<= 1;
        }
    } else {
        kk = -1;
        while (!(w & 0x80000000u)) { /* further zeros of the run */
            kk--;
            w <<= 1;
        }
        w &= 0x7FFFFFFFu; /* drop the terminating one */
    }
    *k = kk;
    *e = (int)(w >> 29);
    *f = ((w << 1) | 0x40000000u) & 0x7FFFFFFFu;
}

/* Pack sign/k/e and a significand whose hidden bit is at bit 62, with the port's
 * rounding (kernel_entry.cl:167-216, 318-367, 487-537):
 *   - the fraction below the hidden bit is shifted right by run+2, and bits that fall
 *     off the 64-bit word are simply lost;
 *   - round to nearest even using bit 31 of the shifted word as the guard bit and
 *     bits 30..0 of that word as the sticky bits -- for every run length, which for
 *     run == 30 leaves the lower exponent bit out of the sticky test;
 *   - |k| beyond the representable range saturates to maxpos / minpos. */
static uint32_t orc_pack(int neg, int k, int e, uint64_t sig62)
{
    uint32_t u;
    int run = (k < 0) ? -k : k + 1;
    if (run > 30) {
        u = (k < 0) ? 0x00000001u : 0x7FFFFFFFu;
    } else {
        uint32_t regime = (k < 0) ? (0x40000000u >> run) : (0x7FFFFFFFu - (0x7FFFFFFFu >> run));
        uint64_t tail = (sig62 & 0x3FFFFFFFFFFFFFFFull) >> (run + 2);
        uint32_t ebits;
        int guard;
        if (run <= 28) {
            ebits = (uint32_t)e << (28 - run);
            guard = (int)((tail >> 31) & 1u);
        } else if (run == 29) {
            ebits = (uint32_t)e >> 1;
            guard = e & 1;
        } else {
            ebits = 0;
            guard = (e >> 1) & 1;
        }
        u = regime + ebits + (uint32_t)(tail >> 32);
        if (guard) {
            int sticky = (tail & 0x7FFFFFFFull) != 0;
            u += (u & 1u) | (uint32_t)sticky;
        }
    }
    return neg ? 0u - u : u;
}

/* Same-sign addition of magnitudes (kernel_entry.cl:88-217). */
static uint32_t orc_add_same(uint32_t a, uint32_t b)
{
    int neg = (int)(a >> 31);
    int ka, ea, kb, eb, shift, k, e;
    uint32_t fa, fb;
    uint64_t sa, sb;
    if (neg) {
        a = 0u - a;
        b = 0u - b;
    }
    if ((int32_t)a < (int32_t)b) {
        uint32_t t = a;
        a = b;
        b = t;
    }
    orc_fields(a, &ka, &ea, &fa);
    orc_fields(b, &kb, &eb, &fb);
    sa = (uint64_t)fa << 32; /* hidden bit at 62 */
    sb = (uint64_t)fb << 32;
    shift = 4 * (ka - kb) + ea - eb;
    sb = (shift > 63) ? 0 : (sb >> shift); /* truncating alignment */
    sa += sb;
    k = ka;
    e = ea;
    if (sa >> 63) { /* carry out of the hidden bit */
        if (++e > 3) {
            k++;
            e = 0;
        }
        sa >>= 1;
    }
    return orc_pack(neg, k, e, sa);
}

/* Opposite-sign addition (kernel_entry.cl:219-368). */
static uint32_t orc_add_diff(uint32_t a, uint32_t b)
{
    int neg = (int)(a >> 31);
    int ka, ea, kb, eb, shift, k, e;
    uint32_t fa, fb;
    uint64_t sa, sb;
    if (neg)
        a = 0u - a;
    else
        b = 0u - b;
    if (a == b)
        return 0; /* exact cancellation */
    if ((int32_t)a < (int32_t)b) {
        uint32_t t = a;
        a = b;
        b = t;
        neg = !neg;
    }
    orc_fields(a, &ka, &ea, &fa);
    orc_fields(b, &kb, &eb, &fb);
    sa = (uint64_t)fa << 32;
    sb = (uint64_t)fb << 32;
    shift = 4 * (ka - kb) + ea - eb;
    if (shift > 63) /* b vanishes entirely: a comes back unchanged */
        return neg ? 0u - a : a;
    sa -= sb >> shift; /* truncating alignment, then exact difference */
    k = ka;
    e = ea;
    while ((sa >> 59) == 0) { /* renormalise a regime step (4 binades) at a time */
        k--;
        sa <<= 4;
    }
    while (!(sa & 0x4000000000000000ull)) { /* then one binade at a time */
        if (e == 0) {
            k--;
            e = 3;
        } else {
            e--;
        }
        sa <<= 1;
    }
    return orc_pack(neg, k, e, sa);
}

/* kernel_entry.cl:370-397: zero short-circuits first (returning a|b), then NaR. */
uint32_t orc_p32_add(uint32_t a, uint32_t b)
{
    if (a == 0 || b == 0)
        return a | b;
    if (a == NAR || b == NAR)
        return NAR;
    return ((a ^ b) >> 31) ? orc_add_diff(a, b) : orc_add_same(a, b);
}

uint32_t orc_p32_neg(uint32_t a) { return 0u - a; }

/* a - b is add(a, -b) in the reference's posit32 class usage. */
uint32_t orc_p32_sub(uint32_t a, uint32_t b) { return orc_p32_add(a, 0u - b); }

/* kernel_entry.cl:399-538: NaR first, then zero; 31x31-bit significand product. */
uint32_t orc_p32_mul(uint32_t a, uint32_t b)
{
    int neg, ka, ea, kb, eb, k, e;
    uint32_t fa, fb;
    uint64_t p;
    if (a == NAR || b == NAR)
        return NAR;
    if (a == 0 || b == 0)
        return 0;
    neg = (int)((a ^ b) >> 31);
    if (a >> 31)
        a = 0u - a;
    if (b >> 31)
        b = 0u - b;
    orc_fields(a, &ka, &ea, &fa);
    orc_fields(b, &kb, &eb, &fb);
    k = ka + kb;
    e = ea + eb;
    p = (uint64_t)fa * fb; /* hidden bit at 60, or 61 after a carry */
    if (e > 3) {
        k++;
        e &= 3;
    }
    if (p >> 61) {
        if (++e > 3) {
            k++;
            e &= 3;
        }
        p >>= 1;
    }
    return orc_pack(neg, k, e, p << 2);
}

uint32_t orc_p32_abs(uint32_t a)
{
    /* util.cpp:12-17: negate when (signed) below zero; NaR stays NaR */
    return ((int32_t)a < 0) ? 0u - a : a;
}

/* Correctly rounded packing (posit standard, round to nearest even on the bit
 * string, never to zero or NaR) of (-1)^neg * 2^scale * sig62/2^62, with `sticky`
 * standing for any nonzero bits below sig62.  sig62 has its hidden bit at bit 62.
 * Used for the operations that have no in-tree reference source. */
static uint32_t orc_pack_exact(int neg, int scale, uint64_t sig62, int sticky)
{
    uint32_t u;
    int k = (scale >= 0) ? scale / 4 : -((-scale + 3) / 4);
    int e = scale - 4 * k;
    if (k >= 30) {
        u = 0x7FFFFFFFu;
    } else if (k < -30) {
        u = 0x00000001u;
    } else {
        int run = (k < 0) ? -k : k + 1; /* 1..30 */
        /* body = regime run + terminator + 2 exponent bits + 62 fraction bits */
        unsigned __int128 body;
        int len = run + 1 + 2 + 62, drop;
        unsigned __int128 rem, half;
        if (k < 0)
            body = 1; /* zeros then a terminating one */
        else
            body = (((unsigned __int128)1 << run) - 1) << 1; /* ones then a zero */
        body = (body << 2) | (unsigned)e;
        body = (body << 62) | (sig62 & 0x3FFFFFFFFFFFFFFFull);
        drop = len - 31;
        rem = body & (((unsigned __int128)1 << drop) - 1);
        half = (unsigned __int128)1 << (drop - 1);
        u = (uint32_t)(body >> drop);
        /* above half, or an exact tie (no sticky) broken towards the even pattern */
        if (rem > half || (rem == half && (sticky || (u & 1u))))
            u += 1;
    }
    return neg ? 0u - u : u;
}

/* Division: correctly rounded (no in-tree source; unpinned vs SoftPosit). */
uint32_t orc_p32_div(uint32_t a, uint32_t b)
{
    int neg, ka, ea, kb, eb, scale;
    uint32_t fa, fb;
    uint64_t num, q, r;
    if (a == NAR || b == NAR || b == 0)
        return NAR;
    if (a == 0)
        return 0;
    neg = (int)((a ^ b) >> 31);
    if (a >> 31)
        a = 0u - a;
    if (b >> 31)
        b = 0u - b;
    orc_fields(a, &ka, &ea, &fa);
    orc_fields(b, &kb, &eb, &fb);
    num = (uint64_t)fa << 32;
    q = num / fb;
    r = num % fb;
    scale = (4 * ka + ea) - (4 * kb + eb);
    if (q >> 32) { /* quotient >= 2: hidden bit at 32 */
        return orc_pack_exact(neg, scale, q << 30, r != 0);
    }
    return orc_pack_exact(neg, scale - 1, q << 31, r != 0);
}

static uint64_t orc_isqrt64(uint64_t x, uint64_t *rem)
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

/* Square root: correctly rounded (no in-tree source; unpinned vs SoftPosit). */
uint32_t orc_p32_sqrt(uint32_t a)
{
    int k, e, scale, odd;
    uint32_t f;
    uint64_t m, r, rem;
    if (a == 0)
        return 0;
    if (a >> 31)
        return NAR; /* negative or NaR */
    orc_fields(a, &k, &e, &f);
    scale = 4 * k + e;
    odd = scale & 1;
    m = (uint64_t)f << odd;         /* value = m/2^30 * 2^(scale-odd) */
    r = orc_isqrt64(m << 32, &rem); /* sqrt(m/2^30) = r/2^31 (+ remainder) */
    return orc_pack_exact(0, (scale - odd) / 2, r << 31, rem != 0);
}

uint32_t orc_p32_from_double(double x)
{
    int ex;
    double m;
    uint64_t sig;
    int neg = 0;
    if (x == 0.0)
        return 0;
    if (isnan(x) || isinf(x))
        return NAR;
    if (x < 0) {
        neg = 1;
        x = -x;
    }
    m = frexp(x, &ex);                 /* x = m * 2^ex, m in [0.5, 1) */
    sig = (uint64_t)ldexp(m, 63);      /* hidden bit at 62, exact (53 bits) */
    return orc_pack_exact(neg, ex - 1, sig, 0);
}

double orc_p32_to_double(uint32_t a)
{
    int k, e, neg;
    uint32_t f;
    if (a == 0)
        return 0.0;
    if (a == NAR)
        return NAN;
    neg = (int)(a >> 31);
    if (neg)
        a = 0u - a;
    orc_fields(a, &k, &e, &f);
    return (neg ? -1.0 : 1.0) * ldexp((double)f, 4 * k + e - 30);
}

void orc_p32_add_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = orc_p32_add(a[i], b[i]);
}

void orc_p32_mul_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = orc_p32_mul(a[i], b[i]);
}

void orc_p32_div_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = orc_p32_div(a[i], b[i]);
}

void orc_p32_sqrt_n(const uint32_t *a, uint32_t *out, int64_t n)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = orc_p32_sqrt(a[i]);
}

void orc_p32_from_double_n(const double *x, uint32_t *out, int64_t n)
{
    int64_t i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = orc_p32_from_double(x[i]);
}

void orc_p32_to_double_n(const uint32_t *a, double *out, int64_t n)
{
    int64_t i;
    for (i = 0; i < n; i++)
        out[i] = orc_p32_to_double(a[i]);
}

/* ------------------------------------------------------------------------- */
/* BLAS                                                                      */
/* ------------------------------------------------------------------------- */

#define A_(i, j) a[(size_t)(i) + (size_t)(j) * (size_t)lda]
#define B_(i, j) b[(size_t)(i) + (size_t)(j) * (size_t)ldb]
#define C_(i, j) c[(size_t)(i) + (size_t)(j) * (size_t)ldc]

static int same(char x, char y) { return toupper((unsigned char)x) == toupper((unsigned char)y); }
static int imax(int x, int y) { return x > y ? x : y; }
static int imin(int x, int y) { return x < y ? x : y; }

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* libRpack/Rgemm.cpp:62-251.  NN/NT: C <- beta*C (0 if beta==0, untouched if
 * beta==1), then c += (alpha*b_lj)*a_il for l ascending.  TN/TT: t = sum_l a_li*b_lj
 * from zero, then c = alpha*t (beta==0) or alpha*t + beta*c. */
int orc_rgemm_cols(char transa, char transb, int m, int n, int k, uint32_t alpha,
                   const uint32_t *a, int lda, const uint32_t *b, int ldb,
                   uint32_t beta, uint32_t *c, int ldc, int j0, int j1)
{
    int nota = same(transa, 'N'), notb = same(transb, 'N');
    int nrowa = nota ? m : k, nrowb = notb ? k : n;
    int j;
    if (!nota && !same(transa, 'C') && !same(transa, 'T'))
        return 1;
    if (!notb && !same(transb, 'C') && !same(transb, 'T'))
        return 2;
    if (m < 0)
        return 3;
    if (n < 0)
        return 4;
    if (k < 0)
        return 5;
    if (lda < imax(1, nrowa))
        return 8;
    if (ldb < imax(1, nrowb))
        return 10;
    if (ldc < imax(1, m))
        return 13;
    if (m == 0 || n == 0 || ((alpha == 0 || k == 0) && beta == ONE))
        return 0;
    if (j0 < 0)
        j0 = 0;
    if (j1 > n)
        j1 = n;
    if (alpha == 0) {
#pragma omp parallel for schedule(static)
        for (j = j0; j < j1; j++)
            for (int i = 0; i < m; i++)
                C_(i, j) = (beta == 0) ? 0u : orc_p32_mul(beta, C_(i, j));
        return 0;
    }
    if (nota) {
        /* scale, then accumulate (Rgemm.cpp:168-185 NN, 210-227 NT) */
#pragma omp parallel for schedule(dynamic, 1)
        for (j = j0; j < j1; j++) {
            if (beta == 0) {
                for (int i = 0; i < m; i++)
                    C_(i, j) = 0;
            } else if (beta != ONE) {
                for (int i = 0; i < m; i++)
                    C_(i, j) = orc_p32_mul(beta, C_(i, j));
            }
            for (int l = 0; l < k; l++) {
                uint32_t t = orc_p32_mul(alpha, notb ? B_(l, j) : B_(j, l));
                for (int i = 0; i < m; i++)
                    C_(i, j) = orc_p32_add(C_(i, j), orc_p32_mul(t, A_(i, l)));
            }
        }
    } else {
        /* dot, then combine (Rgemm.cpp:190-203 TN, 232-245 TT) */
#pragma omp parallel for schedule(dynamic, 1)
        for (j = j0; j < j1; j++) {
            for (int i = 0; i < m; i++) {
                uint32_t t = 0;
                for (int l = 0; l < k; l++)
                    t = orc_p32_add(t, orc_p32_mul(A_(l, i), notb ? B_(l, j) : B_(j, l)));
                if (beta == 0)
                    C_(i, j) = orc_p32_mul(alpha, t);
                else
                    C_(i, j) = orc_p32_add(orc_p32_mul(alpha, t), orc_p32_mul(beta, C_(i, j)));
            }
        }
    }
    return 0;
}

int orc_rgemm(char transa, char transb, int m, int n, int k, uint32_t alpha,
              const uint32_t *a, int lda, const uint32_t *b, int ldb,
              uint32_t beta, uint32_t *c, int ldc)
{
    return orc_rgemm_cols(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 0, n);
}

/* iRamax.cpp:31-88: first index (1-based) of the strict maximum of abs(x). */
int orc_iramax(int n, const uint32_t *x, int incx)
{
    int best = 1, i;
    int32_t dmax;
    if (n < 1 || incx <= 0)
        return 0;
    if (n == 1)
        return 1;
    dmax = (int32_t)orc_p32_abs(x[0]);
    for (i = 1; i < n; i++) {
        int32_t v = (int32_t)orc_p32_abs(x[(size_t)i * incx]);
        if (v > dmax) {
            best = i + 1;
            dmax = v;
        }
    }
    return best;
}

/* Rscal.cpp:62-119: x <- da*x element by element. */
void orc_rscal(int n, uint32_t da, uint32_t *x, int incx)
{
    int i;
    if (n <= 0 || incx <= 0)
        return;
    for (i = 0; i < n; i++)
        x[(size_t)i * incx] = orc_p32_mul(da, x[(size_t)i * incx]);
}

/* Rlaswp.cpp:32-111: sequential row interchanges k1..k2 (reverse order if incx<0);
 * every column sees the same swap sequence, so the 32-column blocking of the
 * reference does not change any value. */
void orc_rlaswp(int n, uint32_t *a, int lda, int k1, int k2, const int *ipiv, int incx)
{
    int i1, i2, inc, ix0, col;
    if (incx > 0) {
        ix0 = k1;
        i1 = k1;
        i2 = k2;
        inc = 1;
    } else if (incx < 0) {
        ix0 = k1 + (k1 - k2) * incx;
        i1 = k2;
        i2 = k1;
        inc = -1;
    } else {
        return;
    }
    for (col = 0; col < n; col++) {
        int ix = ix0, i;
        for (i = i1; inc > 0 ? i <= i2 : i >= i2; i += inc) {
            int ip = ipiv[ix - 1];
            if (ip != i) {
                uint32_t t = A_(i - 1, col);
                A_(i - 1, col) = A_(ip - 1, col);
                A_(ip - 1, col) = t;
            }
            ix += incx;
        }
    }
}

/* Rtrsm.cpp:31-291, all eight side/uplo/trans variants in the reference's order. */
int orc_rtrsm(char side, char uplo, char transa, char diag, int m, int n, uint32_t alpha,
              const uint32_t *a, int lda, uint32_t *b, int ldb)
{
    int lside = same(side, 'L'), upper = same(uplo, 'U'), nounit = same(diag, 'N');
    int notr = same(transa, 'N');
    int nrowa = lside ? m : n;
    int i, j, k;
    if (!lside && !same(side, 'R'))
        return 1;
    if (!upper && !same(uplo, 'L'))
        return 2;
    if (!notr && !same(transa, 'T') && !same(transa, 'C'))
        return 3;
    if (!same(diag, 'U') && !same(diag, 'N'))
        return 4;
    if (m < 0)
        return 5;
    if (n < 0)
        return 6;
    if (lda < imax(1, nrowa))
        return 9;
    if (ldb < imax(1, m))
        return 11;
    if (m == 0 || n == 0)
        return 0;
    if (alpha == 0) {
        for (j = 0; j < n; j++)
            for (i = 0; i < m; i++)
                B_(i, j) = 0;
        return 0;
    }
    if (lside) {
        if (notr) {
            /* B := alpha*inv(A)*B */
            for (j = 0; j < n; j++) {
                if (alpha != ONE)
                    for (i = 0; i < m; i++)
                        B_(i, j) = orc_p32_mul(alpha, B_(i, j));
                if (upper) {
                    for (k = m - 1; k >= 0; k--) {
                        if (B_(k, j) != 0) {
                            if (nounit)
                                B_(k, j) = orc_p32_div(B_(k, j), A_(k, k));
                            for (i = 0; i < k; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(B_(k, j), A_(i, k)));
                        }
                    }
                } else {
                    for (k = 0; k < m; k++) {
                        if (B_(k, j) != 0) {
                            if (nounit)
                                B_(k, j) = orc_p32_div(B_(k, j), A_(k, k));
                            for (i = k + 1; i < m; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(B_(k, j), A_(i, k)));
                        }
                    }
                }
            }
        } else {
            /* B := alpha*inv(A**T)*B */
            for (j = 0; j < n; j++) {
                if (upper) {
                    for (i = 0; i < m; i++) {
                        uint32_t t = orc_p32_mul(alpha, B_(i, j));
                        for (k = 0; k < i; k++)
                            t = orc_p32_sub(t, orc_p32_mul(A_(k, i), B_(k, j)));
                        if (nounit)
                            t = orc_p32_div(t, A_(i, i));
                        B_(i, j) = t;
                    }
                } else {
                    for (i = m - 1; i >= 0; i--) {
                        uint32_t t = orc_p32_mul(alpha, B_(i, j));
                        for (k = i + 1; k < m; k++)
                            t = orc_p32_sub(t, orc_p32_mul(A_(k, i), B_(k, j)));
                        if (nounit)
                            t = orc_p32_div(t, A_(i, i));
                        B_(i, j) = t;
                    }
                }
            }
        }
    } else {
        if (notr) {
            /* B := alpha*B*inv(A) */
            if (upper) {
                for (j = 0; j < n; j++) {
                    if (alpha != ONE)
                        for (i = 0; i < m; i++)
                            B_(i, j) = orc_p32_mul(alpha, B_(i, j));
                    for (k = 0; k < j; k++)
                        if (A_(k, j) != 0)
                            for (i = 0; i < m; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(A_(k, j), B_(i, k)));
                    if (nounit) {
                        uint32_t t = orc_p32_div(ONE, A_(j, j));
                        for (i = 0; i < m; i++)
                            B_(i, j) = orc_p32_mul(t, B_(i, j));
                    }
                }
            } else {
                for (j = n - 1; j >= 0; j--) {
                    if (alpha != ONE)
                        for (i = 0; i < m; i++)
                            B_(i, j) = orc_p32_mul(alpha, B_(i, j));
                    for (k = j + 1; k < n; k++)
                        if (A_(k, j) != 0)
                            for (i = 0; i < m; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(A_(k, j), B_(i, k)));
                    if (nounit) {
                        uint32_t t = orc_p32_div(ONE, A_(j, j));
                        for (i = 0; i < m; i++)
                            B_(i, j) = orc_p32_mul(t, B_(i, j));
                    }
                }
            }
        } else {
            /* B := alpha*B*inv(A**T) */
            if (upper) {
                for (k = n - 1; k >= 0; k--) {
                    if (nounit) {
                        uint32_t t = orc_p32_div(ONE, A_(k, k));
                        for (i = 0; i < m; i++)
                            B_(i, k) = orc_p32_mul(t, B_(i, k));
                    }
                    for (j = 0; j < k; j++)
                        if (A_(j, k) != 0) {
                            uint32_t t = A_(j, k);
                            for (i = 0; i < m; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(t, B_(i, k)));
                        }
                    if (alpha != ONE)
                        for (i = 0; i < m; i++)
                            B_(i, k) = orc_p32_mul(alpha, B_(i, k));
                }
            } else {
                for (k = 0; k < n; k++) {
                    if (nounit) {
                        uint32_t t = orc_p32_div(ONE, A_(k, k));
                        for (i = 0; i < m; i++)
                            B_(i, k) = orc_p32_mul(t, B_(i, k));
                    }
                    for (j = k + 1; j < n; j++)
                        if (A_(j, k) != 0) {
                            uint32_t t = A_(j, k);
                            for (i = 0; i < m; i++)
                                B_(i, j) = orc_p32_sub(B_(i, j), orc_p32_mul(t, B_(i, k)));
                        }
                    if (alpha != ONE)
                        for (i = 0; i < m; i++)
                            B_(i, k) = orc_p32_mul(alpha, B_(i, k));
                }
            }
        }
    }
    return 0;
}

/* Rsyrk.cpp:31-215. */
int orc_rsyrk(char uplo, char trans, int n, int k, uint32_t alpha, const uint32_t *a,
              int lda, uint32_t beta, uint32_t *c, int ldc)
{
    int upper = same(uplo, 'U'), notr = same(trans, 'N');
    int nrowa = notr ? n : k;
    int i, j, l;
    if (!upper && !same(uplo, 'L'))
        return 1;
    if (!notr && !same(trans, 'T') && !same(trans, 'C'))
        return 2;
    if (n < 0)
        return 3;
    if (k < 0)
        return 4;
    if (lda < imax(1, nrowa))
        return 7;
    if (ldc < imax(1, n))
        return 10;
    if (n == 0 || ((alpha == 0 || k == 0) && beta == ONE))
        return 0;
    if (alpha == 0) {
        for (j = 0; j < n; j++) {
            int lo = upper ? 0 : j, hi = upper ? j : n - 1;
            for (i = lo; i <= hi; i++)
                C_(i, j) = (beta == 0) ? 0u : orc_p32_mul(beta, C_(i, j));
        }
        return 0;
    }
    for (j = 0; j < n; j++) {
        int lo = upper ? 0 : j, hi = upper ? j : n - 1;
        if (notr) {
            if (beta == 0) {
                for (i = lo; i <= hi; i++)
                    C_(i, j) = 0;
            } else if (beta != ONE) {
                for (i = lo; i <= hi; i++)
                    C_(i, j) = orc_p32_mul(beta, C_(i, j));
            }
            for (l = 0; l < k; l++) {
                if (A_(j, l) != 0) {
                    uint32_t t = orc_p32_mul(alpha, A_(j, l));
                    for (i = lo; i <= hi; i++)
                        C_(i, j) = orc_p32_add(C_(i, j), orc_p32_mul(t, A_(i, l)));
                }
            }
        } else {
            for (i = lo; i <= hi; i++) {
                uint32_t t = 0;
                for (l = 0; l < k; l++)
                    t = orc_p32_add(t, orc_p32_mul(A_(l, i), A_(l, j)));
                if (beta == 0)
                    C_(i, j) = orc_p32_mul(alpha, t);
                else
                    C_(i, j) = orc_p32_add(orc_p32_mul(alpha, t), orc_p32_mul(beta, C_(i, j)));
            }
        }
    }
    return 0;
}

/* Rgemv.cpp:~40-204 (the residual b = A*x of the drivers). */
int orc_rgemv(char trans, int m, int n, uint32_t alpha, const uint32_t *a, int lda,
              const uint32_t *x, int incx, uint32_t beta, uint32_t *y, int incy)
{
    int notr = same(trans, 'N');
    int lenx, leny, kx, ky, i, j;
    if (!notr && !same(trans, 'T') && !same(trans, 'C'))
        return 1;
    if (m < 0)
        return 2;
    if (n < 0)
        return 3;
    if (lda < imax(1, m))
        return 6;
    if (incx == 0)
        return 8;
    if (incy == 0)
        return 11;
    if (m == 0 || n == 0 || (alpha == 0 && beta == ONE))
        return 0;
    lenx = notr ? n : m;
    leny = notr ? m : n;
    kx = incx > 0 ? 0 : -(lenx - 1) * incx;
    ky = incy > 0 ? 0 : -(leny - 1) * incy;
    if (beta != ONE)
        for (i = 0; i < leny; i++) {
            uint32_t *yy = &y[ky + i * incy];
            *yy = (beta == 0) ? 0u : orc_p32_mul(beta, *yy);
        }
    if (alpha == 0)
        return 0;
    if (notr) {
        for (j = 0; j < n; j++) {
            uint32_t t = orc_p32_mul(alpha, x[kx + j * incx]);
            for (i = 0; i < m; i++) {
                uint32_t *yy = &y[ky + i * incy];
                *yy = orc_p32_add(*yy, orc_p32_mul(t, A_(i, j)));
            }
        }
    } else {
        for (j = 0; j < n; j++) {
            uint32_t t = 0;
            uint32_t *yy = &y[ky + j * incy];
            for (i = 0; i < m; i++)
                t = orc_p32_add(t, orc_p32_mul(A_(i, j), x[kx + i * incx]));
            *yy = orc_p32_add(*yy, orc_p32_mul(alpha, t));
        }
    }
    return 0;
}

/* Rgetrf2.cpp:32-185: recursive LU with partial pivoting.  Returns info
 * (0, or the first zero pivot, 1-based); negative for a bad argument. */
int orc_rgetrf2(int m, int n, uint32_t *a, int lda, int *ipiv)
{
    int info = 0;
    if (m < 0)
        return -1;
    if (n < 0)
        return -2;
    if (lda < imax(1, m))
        return -4;
    if (m == 0 || n == 0)
        return 0;
    if (m == 1) {
        ipiv[0] = 1;
        if (a[0] == 0)
            info = 1;
    } else if (n == 1) {
        /* sfmin = FLT_MIN converts to minpos in posit32 (Rgetrf2.cpp:103) */
        const uint32_t sfmin = orc_p32_from_double(1.17549435082228750797e-38);
        int p = orc_iramax(m, a, 1);
        ipiv[0] = p;
        if (a[p - 1] != 0) {
            int i;
            if (p != 1) {
                uint32_t t = a[0];
                a[0] = a[p - 1];
                a[p - 1] = t;
            }
            if ((int32_t)orc_p32_abs(a[0]) >= (int32_t)sfmin) {
                orc_rscal(m - 1, orc_p32_div(ONE, a[0]), &a[1], 1);
            } else {
                for (i = 1; i < m; i++)
                    a[i] = orc_p32_div(a[i], a[0]);
            }
        } else {
            info = 1;
        }
    } else {
        int n1 = imin(m, n) / 2, n2 = n - n1, iinfo, i;
        iinfo = orc_rgetrf2(m, n1, a, lda, ipiv);
        if (info == 0 && iinfo > 0)
            info = iinfo;
        orc_rlaswp(n2, &A_(0, n1), lda, 1, n1, ipiv, 1);
        orc_rtrsm('L', 'L', 'N', 'U', n1, n2, ONE, a, lda, &A_(0, n1), lda);
        orc_rgemm('N', 'N', m - n1, n2, n1, orc_p32_neg(ONE), &A_(n1, 0), lda, &A_(0, n1), lda,
                  ONE, &A_(n1, n1), lda);
        iinfo = orc_rgetrf2(m - n1, n2, &A_(n1, n1), lda, &ipiv[n1]);
        if (info == 0 && iinfo > 0)
            info = iinfo + n1;
        for (i = n1; i < imin(m, n); i++)
            ipiv[i] += n1;
        orc_rlaswp(n1, a, lda, n1 + 1, imin(m, n), ipiv, 1);
    }
    return info;
}

/* Rgetrf.cpp:32-137 with the block size nb supplied by the caller (the reference
 * takes it from iMlaenv). */
int orc_rgetrf(int m, int n, uint32_t *a, int lda, int *ipiv, int nb)
{
    int info = 0, j, mn = imin(m, n);
    if (m < 0)
        return -1;
    if (n < 0)
        return -2;
    if (lda < imax(1, m))
        return -4;
    if (m == 0 || n == 0)
        return 0;
    if (nb <= 1 || nb >= mn)
        return orc_rgetrf2(m, n, a, lda, ipiv);
    for (j = 0; j < mn; j += nb) {
        int jb = imin(mn - j, nb), i, iinfo;
        iinfo = orc_rgetrf2(m - j, jb, &A_(j, j), lda, &ipiv[j]);
        if (info == 0 && iinfo > 0)
            info = iinfo + j;
        for (i = j; i < imin(m, j + jb); i++)
            ipiv[i] += j;
        orc_rlaswp(j, a, lda, j + 1, j + jb, ipiv, 1);
        if (j + jb < n) {
            orc_rlaswp(n - j - jb, &A_(0, j + jb), lda, j + 1, j + jb, ipiv, 1);
            orc_rtrsm('L', 'L', 'N', 'U', jb, n - j - jb, ONE, &A_(j, j), lda, &A_(j, j + jb), lda);
            if (j + jb < m)
                orc_rgemm('N', 'N', m - j - jb, n - j - jb, jb, orc_p32_neg(ONE), &A_(j + jb, j), lda,
                          &A_(j, j + jb), lda, ONE, &A_(j + jb, j + jb), lda);
        }
    }
    return info;
}

/* Rgetrs.cpp:32-118. */
int orc_rgetrs(char trans, int n, int nrhs, const uint32_t *a, int lda, const int *ipiv,
               uint32_t *b, int ldb)
{
    int notr = same(trans, 'N');
    if (!notr && !same(trans, 'T') && !same(trans, 'C'))
        return -1;
    if (n < 0)
        return -2;
    if (nrhs < 0)
        return -3;
    if (lda < imax(1, n))
        return -5;
    if (ldb < imax(1, n))
        return -8;
    if (n == 0 || nrhs == 0)
        return 0;
    if (notr) {
        orc_rlaswp(nrhs, b, ldb, 1, n, ipiv, 1);
        orc_rtrsm('L', 'L', 'N', 'U', n, nrhs, ONE, a, lda, b, ldb);
        orc_rtrsm('L', 'U', 'N', 'N', n, nrhs, ONE, a, lda, b, ldb);
    } else {
        orc_rtrsm('L', 'U', 'T', 'N', n, nrhs, ONE, a, lda, b, ldb);
        orc_rtrsm('L', 'L', 'T', 'U', n, nrhs, ONE, a, lda, b, ldb);
        orc_rlaswp(nrhs, b, ldb, 1, n, ipiv, -1);
    }
    return 0;
}

/* Rpotrf2.cpp:32-151: recursive Cholesky; a <= 0 (NaR included) fails. */
int orc_rpotrf2(char uplo, int n, uint32_t *a, int lda)
{
    int upper = same(uplo, 'U');
    int n1, n2, iinfo;
    if (!upper && !same(uplo, 'L'))
        return -1;
    if (n < 0)
        return -2;
    if (lda < imax(1, n))
        return -4;
    if (n == 0)
        return 0;
    if (n == 1) {
        if ((int32_t)a[0] <= 0)
            return 1;
        a[0] = orc_p32_sqrt(a[0]);
        return 0;
    }
    n1 = n / 2;
    n2 = n - n1;
    iinfo = orc_rpotrf2(uplo, n1, a, lda);
    if (iinfo != 0)
        return iinfo;
    if (upper) {
        orc_rtrsm('L', 'U', 'T', 'N', n1, n2, ONE, a, lda, &A_(0, n1), lda);
        orc_rsyrk(uplo, 'T', n2, n1, orc_p32_neg(ONE), &A_(0, n1), lda, ONE, &A_(n1, n1), lda);
    } else {
        orc_rtrsm('R', 'L', 'T', 'N', n2, n1, ONE, a, lda, &A_(n1, 0), lda);
        orc_rsyrk(uplo, 'N', n2, n1, orc_p32_neg(ONE), &A_(n1, 0), lda, ONE, &A_(n1, n1), lda);
    }
    iinfo = orc_rpotrf2(uplo, n2, &A_(n1, n1), lda);
    if (iinfo != 0)
        return iinfo + n1;
    return 0;
}

/* Rpotrf.cpp:32-154 with the block size supplied by the caller. */
int orc_rpotrf(char uplo, int n, uint32_t *a, int lda, int nb)
{
    int upper = same(uplo, 'U');
    int j, info = 0;
    if (!upper && !same(uplo, 'L'))
        return -1;
    if (n < 0)
        return -2;
    if (lda < imax(1, n))
        return -4;
    if (n == 0)
        return 0;
    if (nb <= 1 || nb >= n)
        return orc_rpotrf2(uplo, n, a, lda);
    for (j = 0; j < n; j += nb) {
        int jb = imin(nb, n - j);
        uint32_t m1 = orc_p32_neg(ONE);
        if (upper) {
            orc_rsyrk('U', 'T', jb, j, m1, &A_(0, j), lda, ONE, &A_(j, j), lda);
            info = orc_rpotrf2('U', jb, &A_(j, j), lda);
            if (info != 0)
                return info + j;
            if (j + jb < n) {
                orc_rgemm('T', 'N', jb, n - j - jb, j, m1, &A_(0, j), lda, &A_(0, j + jb), lda, ONE,
                          &A_(j, j + jb), lda);
                orc_rtrsm('L', 'U', 'T', 'N', jb, n - j - jb, ONE, &A_(j, j), lda, &A_(j, j + jb), lda);
            }
        } else {
            orc_rsyrk('L', 'N', jb, j, m1, &A_(j, 0), lda, ONE, &A_(j, j), lda);
            info = orc_rpotrf2('L', jb, &A_(j, j), lda);
            if (info != 0)
                return info + j;
            if (j + jb < n) {
                orc_rgemm('N', 'T', n - j - jb, jb, j, m1, &A_(j + jb, 0), lda, &A_(j, 0), lda, ONE,
                          &A_(j + jb, j), lda);
                orc_rtrsm('R', 'L', 'T', 'N', n - j - jb, jb, ONE, &A_(j, j), lda, &A_(j + jb, j), lda);
            }
        }
    }
    return 0;
}

/* Rpotrs.cpp:32-110. */
int orc_rpotrs(char uplo, int n, int nrhs, const uint32_t *a, int lda, uint32_t *b, int ldb)
{
    int upper = same(uplo, 'U');
    if (!upper && !same(uplo, 'L'))
        return -1;
    if (n < 0)
        return -2;
    if (nrhs < 0)
        return -3;
    if (lda < imax(1, n))
        return -5;
    if (ldb < imax(1, n))
        return -7;
    if (n == 0 || nrhs == 0)
        return 0;
    if (upper) {
        orc_rtrsm('L', 'U', 'T', 'N', n, nrhs, ONE, a, lda, b, ldb);
        orc_rtrsm('L', 'U', 'N', 'N', n, nrhs, ONE, a, lda, b, ldb);
    } else {
        orc_rtrsm('L', 'L', 'N', 'N', n, nrhs, ONE, a, lda, b, ldb);
        orc_rtrsm('L', 'L', 'T', 'N', n, nrhs, ONE, a, lda, b, ldb);
    }
    return 0;
}
