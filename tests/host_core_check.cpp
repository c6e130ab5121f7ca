// Host build of the product's posit32 arithmetic (posit_gpu_b200/csrc/posit32.cuh) for
// CPU tests against the oracle.  Compiled by tests/test_posit_core_cpu.py.
#include "../posit_gpu_b200/csrc/posit32.cuh"
#include <stdint.h>
using namespace pg;
extern "C" {
void hc_pmul_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pmul(a[i], b[i]); }
void hc_padd_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = padd(a[i], b[i]); }
void hc_pdiv_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pdiv(a[i], b[i]); }
void hc_psqrt_n(const uint32_t *a, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = psqrt(a[i]); }
void hc_from_double_n(const double *x, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = p32_from_double(x[i]); }
// c + t*a through the decoded fast path (with its exact fallback); counts fast-path steps
long hc_dmac_n(const uint32_t *c, const uint32_t *t, const uint32_t *a, uint32_t *o, long n)
{
    long fast = 0;
    for (long i = 0; i < n; i++) {
        dp32 dc = decode(c[i]), dt = decode(t[i]), da = decode(a[i]), p, r;
        bool ok = dmul_fast(dt, da, p);
        ok = dadd_fast(dc, p, r) && ok;
        fast += ok;
        o[i] = encode(dmac(dc, dt, da));
    }
    return fast;
}
// a chain c <- c + t_l*a_l kept in the decoded domain for len steps
void hc_chain(const uint32_t *c0, const uint32_t *t, const uint32_t *a, uint32_t *o, long nchains, long len)
{
    for (long j = 0; j < nchains; j++) {
        dp32 c = decode(c0[j]);
        for (long l = 0; l < len; l++)
            c = dmac(c, decode(t[j * len + l]), decode(a[j * len + l]));
        o[j] = encode(c);
    }
}
}
