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
}
