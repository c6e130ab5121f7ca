// Host build of the product's posit32 arithmetic (posit_gpu_b200/csrc/posit32.cuh) for
// CPU tests against the oracle.  Compiled by tests/test_posit_core_cpu.py.
#include "../posit_gpu_b200/csrc/posit32.cuh"
#include <stdint.h>
using namespace pg;
static RegimeEntry g_table[RT_N];
static const RegimeEntry *table()
{
    static bool built = false;
    if (!built) {
        for (int i = 0; i < RT_N; i++)
            g_table[i] = regime_entry(RT_MIN + i);
        built = true;
    }
    return g_table - RT_MIN;
}
extern "C" {
void hc_pmul_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pmul(a[i], b[i]); }
void hc_padd_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = padd(a[i], b[i]); }
void hc_pdiv_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pdiv(a[i], b[i]); }
void hc_psqrt_n(const uint32_t *a, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = psqrt(a[i]); }
void hc_from_double_n(const double *x, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = p32_from_double(x[i]); }
// c + t*a through the decoded fast path (with its exact fallback); counts fast-path steps
long hc_dmac_n(const uint32_t *c, const uint32_t *t, const uint32_t *a, uint32_t *o, long n)
{
    // NaR operands are handled outside the decoded domain by the GEMM kernels (flags);
    // here they take the exact path directly.
    const RegimeEntry *tb = table();
    long fast = 0;
    for (long i = 0; i < n; i++) {
        if (c[i] == P32_NAR || t[i] == P32_NAR || a[i] == P32_NAR) {
            o[i] = padd(c[i], pmul(t[i], a[i]));
            continue;
        }
        dp32 dc = decode_gemm(c[i]), dt = decode_gemm(t[i]), da = decode_gemm(a[i]), p, r;
        uint32_t bm, ba;
        dmul_fast(dt, da, tb, p, bm);
        dadd_fast(dc, p, tb, r, ba);
        fast += !((bm | ba) & 0x40000000u);
        o[i] = encode(dmac(dc, dt, da, tb));
    }
    return fast;
}
// a chain c <- c + t_l*a_l kept in the decoded domain for len steps
void hc_chain(const uint32_t *c0, const uint32_t *t, const uint32_t *a, uint32_t *o, long nchains, long len)
{
    const RegimeEntry *tb = table();
    for (long j = 0; j < nchains; j++) {
        dp32 c = decode_gemm(c0[j]);
        for (long l = 0; l < len; l++)
            c = dmac(c, decode_gemm(t[j * len + l]), decode_gemm(a[j * len + l]), tb);
        o[j] = encode(c);
    }
}
// c + t*a through the triangular-solve chain step (computed regime entries; NaR outside)
void hc_dmac_chain_n(const uint32_t *c, const uint32_t *t, const uint32_t *a, uint32_t *o, long n)
{
    for (long i = 0; i < n; i++) {
        if (c[i] == P32_NAR || t[i] == P32_NAR || a[i] == P32_NAR) {
            o[i] = P32_NAR;
            continue;
        }
        o[i] = encode(dmac_chain(decode_gemm(c[i]), decode_gemm(t[i]), decode_gemm(a[i])));
    }
}
// one right-hand side of the L^T solve (trsm_chain.cuh's loop, on the host)
void hc_llt_solve(const uint32_t *L, long ld, uint32_t *b, int m)
{
    for (int i = m - 1; i >= 0; --i) {
        const uint32_t *li = L + (long)i * ld;
        const uint32_t bi = b[i];
        uint32_t nar = bi == P32_NAR;
        dp32 c = decode_gemm(nar ? 0u : bi);
        for (int k = i + 1; k < m; ++k) {
            const uint32_t l = li[k], bk = b[k];
            nar |= (l == P32_NAR) | (bk == P32_NAR);
            c = dmac_chain(c, decode_gemm(bk == P32_NAR ? 0u : 0u - bk), decode_gemm(l == P32_NAR ? 0u : l));
        }
        uint32_t t = nar ? P32_NAR : encode(c);
        b[i] = pdiv(t, li[i]);
    }
}
}
