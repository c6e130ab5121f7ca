// Host build of the product's posit32 arithmetic (posit_gpu_b200/csrc/posit32.cuh) for
// CPU tests against the oracle.  Compiled by tests/test_posit_core_cpu.py.
#include "../posit_gpu_b200/csrc/posit32.cuh"
#include "../posit_gpu_b200/csrc/trsm_chain.cuh"
#include "../posit_gpu_b200/csrc/posit32_div.cuh"
#include <stdint.h>
#include <algorithm>
#include <vector>
using namespace pg;
extern "C" {
void hc_pmul_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pmul(a[i], b[i]); }
void hc_padd_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = padd(a[i], b[i]); }
void hc_pdiv_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pdiv(a[i], b[i]); }
void hc_psqrt_n(const uint32_t *a, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = psqrt(a[i]); }
void hc_pdiv_est_n(const uint32_t *a, const uint32_t *b, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = pdiv_est(a[i], b[i]); }
void hc_psqrt_est_n(const uint32_t *a, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = psqrt_est(a[i]); }
void hc_from_double_n(const double *x, uint32_t *o, long n) { for (long i = 0; i < n; i++) o[i] = p32_from_double(x[i]); }
// c + t*a through the decoded integer form (computed regime entries, exact fallback), as
// llt_chain runs it; counts the steps the fast path did alone
long hc_dmac_n(const uint32_t *c, const uint32_t *t, const uint32_t *a, uint32_t *o, long n)
{
    // NaR operands are handled outside the decoded domain (flags); here they take the
    // exact path directly.
    long fast = 0;
    for (long i = 0; i < n; i++) {
        if (c[i] == P32_NAR || t[i] == P32_NAR || a[i] == P32_NAR) {
            o[i] = padd(c[i], pmul(t[i], a[i]));
            continue;
        }
        dp32 dc = decode_dz(c[i]), dt = decode_dz(t[i]), da = decode_dz(a[i]), p, r;
        uint32_t bm, ba;
        dmul_core(dt, da, ComputedEntry{}, p, bm);
        dadd_core(dc, p, ComputedEntry{}, r, ba);
        fast += !((bm | ba) & 0x40000000u);
        o[i] = encode(dmac_chain(dc, dt, da));
    }
    return fast;
}
// a chain c <- c + t_l*a_l kept in the decoded domain for len steps
void hc_chain(const uint32_t *c0, const uint32_t *t, const uint32_t *a, uint32_t *o, long nchains, long len)
{
    for (long j = 0; j < nchains; j++) {
        dp32 c = decode_dz(c0[j]);
        for (long l = 0; l < len; l++)
            c = dmac_chain(c, decode_dz(t[j * len + l]), decode_dz(a[j * len + l]));
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
        o[i] = encode(dmac_chain(decode_dz(c[i]), decode_dz(t[i]), decode_dz(a[i])));
    }
}
// one right-hand side of the L^T solve: trsm_chain.cuh's llt_chain, built for the host
void hc_llt_solve(const uint32_t *L, long ld, uint32_t *b, int m) { llt_chain(L, (size_t)ld, b, m, false); }
// the same chain run forwards on an upper triangle: U^T solve (Rgetrs 'T', Rpotrs 'U')
void hc_utt_solve(const uint32_t *U, long ld, uint32_t *b, int m, int unit)
{
    llt_chain(U, (size_t)ld, b, m, unit != 0, true);
}
// decode_dz_bf against decode_dz on n patterns (NaR skipped); returns mismatches
long hc_decode_bf_mismatch(const uint32_t *u, long n)
{
    long bad = 0;
    for (long i = 0; i < n; i++) {
        if (u[i] == P32_NAR)
            continue;
        const dp32 a = decode_dz(u[i]), b = decode_dz_bf(u[i]);
        bad += (a.s != b.s) | (a.g != b.g) | (a.x != b.x);
    }
    return bad;
}
// the split L^T solve (products as llt_term, additions as chain_add_run), row by row
void hc_llt_solve_split(const uint32_t *L, long ld, uint32_t *b, int m)
{
    double *q = new double[m > 0 ? m : 1];
    for (int i = m - 1; i >= 0; --i) {
        const uint32_t *li = L + (long)i * ld;
        uint32_t nar = b[i] == P32_NAR;
        for (int k = i + 1; k < m; ++k)
            q[k] = llt_term(li[k], b[k], &nar);
        double c = p32_to_double(b[i] == P32_NAR ? 0u : b[i]);
        if (i + 1 < m) {
            c = chain_add_run(c, q + i + 1, 1);
            c = chain_add_run(c, q + i + 2, m - i - 2);
        }
        uint32_t t = nar ? P32_NAR : p32_from_double(c);
        b[i] = pdiv(t, li[i]);
    }
    delete[] q;
}
// chain_add_run over n terms from patterns (NaR excluded by the caller)
uint32_t hc_chain_add(uint32_t c0, const uint32_t *q, int n)
{
    double *d = new double[n > 0 ? n : 1];
    for (int k = 0; k < n; ++k)
        d[k] = p32_to_double(q[k]);
    uint32_t r = p32_from_double(chain_add_run(p32_to_double(c0), d, n));
    delete[] d;
    return r;
}
// single FP64 chain steps t + q (with their exact fallback) on n pairs; returns the number
// of steps the FP64 form handed to the exact path
long hc_f64_add_n(const uint32_t *t, const uint32_t *q, uint32_t *o, long n)
{
    long flagged = 0;
    for (long i = 0; i < n; i++) {
        uint32_t bad = 0;
        const double r = f64_posit_add(p32_to_double(t[i]), p32_to_double(q[i]), bad);
        flagged += (bad & 0x40000000u) != 0;
        o[i] = p32_from_double((bad & 0x40000000u) ? f64_posit_add_exact(p32_to_double(t[i]), p32_to_double(q[i])) : r);
    }
    return flagged;
}
// c + t*a through the FP64 step (with its exact fallback) on n triples, the rounding
// constants from a table (use_table) or computed; returns the number of steps handed to
// the exact path.  NaR operands are handled outside (flags) by the GEMM.
static uint32_t g_ctab[F64_CONST_ENTRIES];
static void fill_ctab()
{
    for (int e = 0; e < F64_CONST_ENTRIES; e++)
        g_ctab[e] = f64_round_const_top((uint32_t)e);
}
long hc_f64_mac_n(const uint32_t *c, const uint32_t *t, const uint32_t *a, uint32_t *o, long n, int use_table)
{
    fill_ctab();
    long flagged = 0;
    for (long i = 0; i < n; i++) {
        if (c[i] == P32_NAR || t[i] == P32_NAR || a[i] == P32_NAR) {
            o[i] = padd(c[i], pmul(t[i], a[i]));
            continue;
        }
        const double dc = p32_to_double(c[i]), dt = p32_to_double(t[i]), da = p32_to_double(a[i]);
        bool bad;
        const double r = use_table ? f64_posit_mac(dc, dt, da, F64ConstTable{g_ctab}, bad)
                                   : f64_posit_mac(dc, dt, da, F64ConstComputed{}, bad);
        flagged += bad;
        o[i] = p32_from_double(bad ? f64_posit_mac_exact(dc, dt, da) : r);
    }
    return flagged;
}
// Pairs (t, a) whose FP64 product lies exactly on a posit rounding tie while being inexact
// -- the one product case the FP64 step must hand to the exact path.  Random search.
long hc_find_tie_products(uint64_t seed, long tries, uint32_t *t_out, uint32_t *a_out, long max_out)
{
    uint64_t x = seed | 1;
    long found = 0;
    for (long i = 0; i < tries && found < max_out; i++) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        const uint32_t ut = (uint32_t)(0x40000000u | ((x >> 8) & 0x07FFFFFFu)); // [1, 2): 27 fraction bits
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        const uint32_t ua = (uint32_t)(0x40000000u | ((x >> 8) & 0x07FFFFFFu));
        const double dt = p32_to_double(ut), da = p32_to_double(ua);
        const double p = dt * da, e = __builtin_fma(dt, da, -p);
        if (e == 0.0)
            continue;
        const int32_t ep = (int32_t)((f64_bits(p) >> 52) & 0x7FF);
        const uint32_t hp = f64_round_const_hi(ep);
        const double C = f64_from_bits((uint64_t)hp << 32);
        const double q = (p + C) - C;
        const double hulp = f64_from_bits((uint64_t)((hp & 0xFFF00000u) - (53u << 20)) << 32);
        if (p - q == hulp || p - q == -hulp) {
            t_out[found] = ut;
            a_out[found] = ua;
            found++;
        }
    }
    return found;
}
// chains c <- c + t_l*a_l through the GEMM kernels' FP64 step (per-binade constants from
// the table, exact fixups), as the kernels run them; returns the number of fixups
long hc_f64_gemm_chains(const uint32_t *c0, const uint32_t *t, const uint32_t *a, uint32_t *o, long nchains, long len)
{
    fill_ctab();
    long fixes = 0;
    for (long j = 0; j < nchains; j++) {
        double c = p32_to_double(c0[j]);
        for (long l = 0; l < len; l++) {
            const double dt = p32_to_double(t[j * len + l]), da = p32_to_double(a[j * len + l]);
            bool bad;
            const double r = f64_posit_mac(c, dt, da, F64ConstTable{g_ctab}, bad);
            if (bad) {
                c = f64_posit_mac_exact(c, dt, da);
                fixes++;
            } else {
                c = r;
            }
        }
        o[j] = p32_from_double(c);
    }
    return fixes;
}

// One row's chain t + q_0 + ... + q_{len-1} the way lapack.cu's group_chain_scan runs it,
// written out sequentially: one warp takes a window of
// the next 32*E terms, E per lane; each lane's composed map, the exclusive prefix over
// lanes, every lane's walk from its true start, the first invalid step of the window;
// the window advances past it by one exact step (or past its end); a window that ended
// within 64 addends is followed by 32 sequential steps.
static double scan_row_emul(double t, const double *q, int len, int E, long *segs, long *exact)
{
    constexpr int LANES = 32;
    SegFn start[LANES];
    int pos = 0;
    while (pos < len) {
        SegParams sp;
        if (!seg_begin(t, sp)) {
            t = chain_add_one(t, q[pos]);
            ++pos;
            ++*exact;
            continue;
        }
        ++*segs;
        const int end = std::min(len, pos + LANES * E);
        SegFn acc = {0, 0};
        for (int l = 0; l < LANES; ++l) {
            start[l] = acc;
            SegFn f = {0, 0};
            const int j0 = pos + l * E, j1 = std::min(j0 + E, end);
            for (int j = j0; j < j1; ++j) {
                int32_t K;
                bool r;
                f = seg_then(f, seg_fn(q[j], sp, K, r));
            }
            acc = seg_then(acc, f);
        }
        uint64_t key = ~0ull;
        int32_t Mend = 0;
        for (int l = 0; l < LANES; ++l) {
            const int j0 = pos + l * E, j1 = std::min(j0 + E, end);
            int32_t M = seg_apply(start[l], sp.M0);
            for (int j = j0; j < j1; ++j) {
                int32_t K;
                bool r;
                const SegFn f = seg_fn(q[j], sp, K, r);
                if (!seg_valid(M, K, r, sp)) {
                    key = std::min(key, ((uint64_t)j << 32) | (uint32_t)M);
                    break;
                }
                M = seg_apply(f, M);
            }
            if (j1 == end && j0 < end)
                Mend = M;
        }
        if (key == ~0ull) {
            t = sp.us * (double)Mend;
            pos = end;
        } else {
            const int js = (int)(key >> 32);
            t = chain_add_one(sp.us * (double)(int32_t)(uint32_t)key, q[js]);
            const bool cut_short = js - pos < 64; // lapack.cu: LLT_SHORT_WINDOW, LLT_SEQ_STEPS
            pos = js + 1;
            ++*exact;
            if (cut_short) {
                const int cnt = std::min(32, len - pos);
                t = chain_add_run_reg(t, TermsF64{q + pos}, cnt);
                pos += cnt;
            }
        }
    }
    return t;
}

// The L^T solve with rows summed by scan_row_emul; stats[0] += scans, stats[1] += exact steps.
void hc_llt_solve_scan(const uint32_t *L, long ld, uint32_t *b, int m, int E, long *stats)
{
    std::vector<double> q(m > 0 ? m : 1);
    for (int i = m - 1; i >= 0; --i) {
        const uint32_t *li = L + (long)i * ld;
        uint32_t nar = b[i] == P32_NAR;
        const int len = m - 1 - i;
        for (int j = 0; j < len; ++j)
            q[j] = llt_term(li[i + 1 + j], b[i + 1 + j], &nar);
        const double c = scan_row_emul(p32_to_double(b[i] == P32_NAR ? 0u : b[i]), q.data(), len, E,
                                       &stats[0], &stats[1]);
        uint32_t t = nar ? P32_NAR : p32_from_double(c);
        b[i] = pdiv(t, li[i]);
    }
}
// p32_from_double_exact(p32_to_double(u)) == u over n patterns; returns mismatches
long hc_from_double_exact_mismatch(const uint32_t *u, long n)
{
    long bad = 0;
    for (long i = 0; i < n; i++)
        bad += p32_from_double_exact(p32_to_double(u[i])) != u[i];
    return bad;
}
// Veltkamp's split (the high part of (2^sh+1)s) against rounding the FP64 significand to
// 53 - sh bits with integer operations (nearest, ties to even), for sh = 25..51 on n random
// values per sh, a third of them exact ties and a third one unit either side of a tie.
// Returns the number of mismatches.
long hc_split_round_check(uint64_t seed, long n)
{
    uint64_t st = seed | 1;
    auto rnd = [&]() { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return st; };
    long bad = 0;
    for (int sh = 25; sh <= 51; ++sh) {
        const double C = f64_add(f64_from_bits((uint64_t)(sh + 1023) << 52), 1.0);
        const uint64_t half = (uint64_t)1 << (sh - 1), low = ((uint64_t)1 << sh) - 1;
        for (long i = 0; i < n; ++i) {
            uint64_t m = rnd() & 0xFFFFFFFFFFFFFull;
            const uint64_t kind = rnd() % 4;
            if (kind == 0)
                m = (m & ~low) | half;
            else if (kind == 1)
                m = (m & ~low) | (half + 1);
            else if (kind == 2)
                m = (m & ~low) | (half - 1);
            const uint64_t b = ((rnd() & 1) << 63) | ((uint64_t)(1023 + (int)(rnd() % 241) - 120) << 52) | m;
            const double s = f64_from_bits(b);
            const uint64_t want = (b + (half - 1) + ((b >> sh) & 1)) & ~low;
            const double g = f64_mul(C, s);
            const double r = f64_add(g, f64_add(s, -g));
            bad += f64_bits(r) != want;
        }
    }
    return bad;
}
// The cluster LU panel (lapack.cu, lu_panel_cluster_kernel) restated on the host with the
// same FP64 steps and rounding-constant table: rows stay in their slots, an interchange
// swaps the logical row numbers two slots hold, the pivot is the largest key with the lowest
// logical row among equal keys, and a zero pivot below row k trades back the two slots'
// column-k values.  P is M x jb, column-major with ld M; ipiv receives 1-based pivots;
// returns info (the first zero pivot, 1-based, or 0).
int hc_lu_panel_relabel(uint32_t *P, int M, int jb, int *ipiv)
{
    std::vector<uint32_t> tab(F64_CONST_ENTRIES);
    for (int i = 0; i < F64_CONST_ENTRIES; ++i)
        tab[i] = f64_round_const_top((uint32_t)i);
    const F64ConstTable cof{tab.data()};
    std::vector<double> S((size_t)M * jb); // slot s, column c at S[s * jb + c]
    std::vector<int> row(M);
    for (int s = 0; s < M; ++s) {
        row[s] = s;
        for (int c = 0; c < jb; ++c)
            S[(size_t)s * jb + c] = p32_to_double(P[s + (size_t)c * M]);
    }
    int info = 0;
    std::vector<double> u(jb > 0 ? jb : 1);
    for (int k = 0; k < jb; ++k) {
        int ws = -1, br = -1;
        double bk = -2.0, bv = 0.0;
        for (int s = 0; s < M; ++s)
            if (row[s] >= k) {
                const double v = S[(size_t)s * jb + k], key = v != v ? -1.0 : (v < 0 ? -v : v);
                if (br < 0 || key > bk || (key == bk && row[s] < br)) {
                    bk = key;
                    bv = v;
                    br = row[s];
                    ws = s;
                }
            }
        const int p = br;
        const uint32_t piv = p32_from_double_exact(bv);
        for (int c = k + 1; c < jb; ++c)
            u[c] = -S[(size_t)ws * jb + c];
        int mode = 0;
        uint32_t recip = 0;
        if (piv == 0) {
            if (info == 0)
                info = k + 1;
        } else if ((int32_t)pabs(piv) >= 1) {
            mode = 1;
            recip = pdiv_est(P32_ONE, piv);
        } else {
            mode = 2;
        }
        ipiv[k] = p + 1;
        if (p != k) {
            if (piv == 0)
                for (int s = 0; s < M; ++s)
                    if (row[s] == k) {
                        S[(size_t)ws * jb + k] = S[(size_t)s * jb + k];
                        S[(size_t)s * jb + k] = bv;
                    }
            for (int s = 0; s < M; ++s)
                row[s] = row[s] == k ? p : (row[s] == p ? k : row[s]);
        }
        const double drecip = p32_to_double(recip);
        for (int s = 0; s < M; ++s)
            if (row[s] > k) {
                double *rw = &S[(size_t)s * jb];
                const double dl = mode == 1   ? f64_posit_mul_checked(rw[k], drecip, cof)
                                  : mode == 2 ? p32_to_double(pdiv_est(p32_from_double_exact(rw[k]), piv))
                                              : rw[k];
                rw[k] = dl;
                for (int c = k + 1; c < jb; ++c)
                    rw[c] = f64_posit_mac_checked(rw[c], u[c], dl, cof);
            }
    }
    for (int s = 0; s < M; ++s)
        for (int c = 0; c < jb; ++c)
            P[row[s] + (size_t)c * M] = p32_from_double_exact(S[(size_t)s * jb + c]);
    return info;
}
// The cluster Cholesky panel (lapack.cu, chol_panel_cluster_kernel) restated on the host
// with the same FP64 steps: per column, l_kk = sqrt(a_kk) and 1/l_kk from the holder of row
// k (a_kk <= 0 or NaR stops with info), the column below scaled by 1/l_kk (the FP64 product
// step), then each row's entries up to the diagonal block's edge updated.  P is M x jb
// (M >= jb), column-major with ld M; returns info.
int hc_chol_panel(uint32_t *P, int M, int jb)
{
    std::vector<uint32_t> tab(F64_CONST_ENTRIES);
    for (int i = 0; i < F64_CONST_ENTRIES; ++i)
        tab[i] = f64_round_const_top((uint32_t)i);
    const F64ConstTable cof{tab.data()};
    std::vector<double> S((size_t)M * jb);
    for (int i = 0; i < M; ++i)
        for (int c = 0; c < jb; ++c)
            S[(size_t)i * jb + c] = p32_to_double(P[i + (size_t)c * M]);
    int info = 0;
    std::vector<double> l(jb > 0 ? jb : 1);
    for (int k = 0; k < jb; ++k) {
        const uint32_t akk = p32_from_double_exact(S[(size_t)k * jb + k]);
        if ((int32_t)akk <= 0) {
            info = k + 1;
            break;
        }
        const uint32_t lkk = psqrt_est(akk);
        S[(size_t)k * jb + k] = p32_to_double(lkk);
        const double drecip = p32_to_double(pdiv_est(P32_ONE, lkk));
        for (int i = k + 1; i < M; ++i)
            S[(size_t)i * jb + k] = f64_posit_mul_checked(S[(size_t)i * jb + k], drecip, cof);
        for (int c = k + 1; c < jb; ++c)
            l[c] = -S[(size_t)c * jb + k];
        for (int i = k + 1; i < M; ++i) {
            double *rw = &S[(size_t)i * jb];
            const int cend = i < jb - 1 ? i : jb - 1;
            for (int c = k + 1; c <= cend; ++c)
                rw[c] = f64_posit_mac_checked(rw[c], l[c], rw[k], cof);
        }
    }
    for (int i = 0; i < M; ++i)
        for (int c = 0; c < jb; ++c)
            P[i + (size_t)c * M] = p32_from_double_exact(S[(size_t)i * jb + c]);
    return info;
}
// chain_add_run_reg against chain_add_run on one chain of n terms (patterns); 1 on a match
int hc_chain_reg_check(uint32_t c0, const uint32_t *qp, int n)
{
    std::vector<double> q(n > 0 ? n : 1);
    for (int k = 0; k < n; ++k)
        q[k] = p32_to_double(qp[k]);
    const double a = chain_add_run(p32_to_double(c0), q.data(), n);
    const double b = chain_add_run_reg(p32_to_double(c0), TermsF64{q.data()}, n);
    return p32_from_double(a) == p32_from_double(b);
}
// scan_row_emul against chain_add_run on one chain of n terms (patterns); returns 1 on a match
int hc_scan_row_check(uint32_t c0, const uint32_t *qp, int n, int E, long *stats)
{
    std::vector<double> q(n > 0 ? n : 1);
    for (int k = 0; k < n; ++k)
        q[k] = p32_to_double(qp[k]);
    const double a = chain_add_run(p32_to_double(c0), q.data(), n);
    const double b = scan_row_emul(p32_to_double(c0), q.data(), n, E, &stats[0], &stats[1]);
    return p32_from_double(a) == p32_from_double(b);
}
}
