"""The product's posit32 arithmetic (the same header the CUDA kernels compile),
built for the host, against the oracle: pattern-level ops, conversions, and the
decoded-domain multiply-add fast path of the GEMM inner loop."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
U32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
F64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
I64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
I32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def hc(tmp_path_factory):
    out = tmp_path_factory.mktemp("hc") / "libhc.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", str(out),
                           os.path.join(HERE, "host_core_check.cpp")])
    lib = ctypes.CDLL(str(out))
    for nm in ("hc_pmul_n", "hc_padd_n", "hc_pdiv_n", "hc_pdiv_est_n"):
        getattr(lib, nm).argtypes = [U32, U32, U32, ctypes.c_long]
    lib.hc_psqrt_n.argtypes = [U32, U32, ctypes.c_long]
    lib.hc_psqrt_est_n.argtypes = [U32, U32, ctypes.c_long]
    lib.hc_from_double_n.argtypes = [F64, U32, ctypes.c_long]
    lib.hc_dmac_n.argtypes = [U32, U32, U32, U32, ctypes.c_long]
    lib.hc_dmac_n.restype = ctypes.c_long
    lib.hc_chain.argtypes = [U32, U32, U32, U32, ctypes.c_long, ctypes.c_long]
    lib.hc_dmac_chain_n.argtypes = [U32, U32, U32, U32, ctypes.c_long]
    lib.hc_llt_solve.argtypes = [U32, ctypes.c_long, U32, ctypes.c_int]
    lib.hc_utt_solve.argtypes = [U32, ctypes.c_long, U32, ctypes.c_int, ctypes.c_int]
    lib.hc_llt_solve_split.argtypes = [U32, ctypes.c_long, U32, ctypes.c_int]
    lib.hc_llt_solve_scan.argtypes = [U32, ctypes.c_long, U32, ctypes.c_int, ctypes.c_int, I64]
    lib.hc_scan_row_check.argtypes = [ctypes.c_uint32, U32, ctypes.c_int, ctypes.c_int, I64]
    lib.hc_from_double_exact_mismatch.argtypes = [U32, ctypes.c_long]
    lib.hc_from_double_exact_mismatch.restype = ctypes.c_long
    lib.hc_chain_reg_check.argtypes = [ctypes.c_uint32, U32, ctypes.c_int]
    lib.hc_chain_add.argtypes = [ctypes.c_uint32, U32, ctypes.c_int]
    lib.hc_chain_add.restype = ctypes.c_uint32
    lib.hc_f64_add_n.argtypes = [U32, U32, U32, ctypes.c_long]
    lib.hc_f64_add_n.restype = ctypes.c_long
    lib.hc_f64_mac_n.argtypes = [U32, U32, U32, U32, ctypes.c_long, ctypes.c_int]
    lib.hc_f64_mac_n.restype = ctypes.c_long
    lib.hc_find_tie_products.argtypes = [ctypes.c_uint64, ctypes.c_long, U32, U32, ctypes.c_long]
    lib.hc_find_tie_products.restype = ctypes.c_long
    lib.hc_f64_gemm_chains.argtypes = [U32, U32, U32, U32, ctypes.c_long, ctypes.c_long]
    lib.hc_f64_gemm_chains.restype = ctypes.c_long
    lib.hc_decode_bf_mismatch.argtypes = [U32, ctypes.c_long]
    lib.hc_decode_bf_mismatch.restype = ctypes.c_long
    return lib


def _mix(rng, n):
    """Random patterns, U[-1,1], wide range, long regimes, specials."""
    parts = [rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32),
             oracle.from_double(rng.uniform(-1, 1, n)),
             oracle.from_double((10.0 ** rng.uniform(-20, 20, n)) * np.where(rng.integers(0, 2, n) == 1, -1, 1)),
             (rng.integers(0, 4096, n).astype(np.uint32) ^ (rng.integers(0, 2, n).astype(np.uint32) * 0x7FFFFFFF)),
             np.array([0, 0x80000000, 1, 0x7FFFFFFF, 0xFFFFFFFF, 0x80000001, 0x40000000] * (n // 7 + 1),
                      dtype=np.uint32)[:n]]
    x = np.concatenate(parts)
    rng.shuffle(x)
    return x


def test_pattern_ops_match_oracle(hc):
    rng = np.random.default_rng(1)
    a, b = _mix(rng, 200_000), _mix(rng, 200_000)
    for f_hc, f_or in ((hc.hc_pmul_n, oracle.orc.orc_p32_mul_n), (hc.hc_padd_n, oracle.orc.orc_p32_add_n),
                       (hc.hc_pdiv_n, oracle.orc.orc_p32_div_n)):
        o1, o2 = np.empty_like(a), np.empty_like(a)
        f_hc(a, b, o1, a.size)
        f_or(a, b, o2, a.size)
        assert np.array_equal(o1, o2), f_hc.__name__
    o1, o2 = np.empty_like(a), np.empty_like(a)
    hc.hc_psqrt_n(a, o1, a.size)
    oracle.orc.orc_p32_sqrt_n(a, o2, a.size)
    assert np.array_equal(o1, o2)


def test_division_and_root_from_fp64_estimates_match_oracle(hc):
    """pdiv_est / psqrt_est (the integer quotient and root from one FP64 division or square
    root, corrected by the exact remainder) equal p32_div / p32_sqrt on mixed patterns, on
    exact quotients (a = b, a = b*c with small c, powers of two), on every significand
    pattern with a fixed scale (square roots near the top and bottom of their binades), and
    on the extremes."""
    rng = np.random.default_rng(11)
    a, b = _mix(rng, 400_000), _mix(rng, 400_000)
    small = oracle.from_double(rng.choice([1.0, 2.0, 3.0, 0.5, 0.75, 1.5, 5.0, 7.0, 0.125], 100_000))
    b2 = _mix(rng, 100_000)
    a2 = np.empty_like(b2)
    oracle.orc.orc_p32_mul_n(b2, small, a2, b2.size)
    a = np.concatenate([a, a2, b2, b2 ^ np.uint32(0x80000000)])
    b = np.concatenate([b, b2, b2, b2])
    o1, o2 = np.empty_like(a), np.empty_like(a)
    hc.hc_pdiv_est_n(a, b, o1, a.size)
    oracle.orc.orc_p32_div_n(a, b, o2, a.size)
    assert np.array_equal(o1, o2)
    # square roots: random patterns, every fraction of the binades [1, 4) and [2^-40, 2^-38)
    fr = np.arange(0, 1 << 22, dtype=np.uint32)
    sq = np.concatenate([_mix(rng, 400_000), 0x40000000 + (fr << 5), 0x40000000 - (fr << 5),
                         np.array([1, 2, 3, 0x7FFFFFFF, 0x7FFFFFFE, 0x40000000, 0x3FFFFFFF], np.uint32)])
    sq = np.ascontiguousarray(sq)
    o1, o2 = np.empty_like(sq), np.empty_like(sq)
    hc.hc_psqrt_est_n(sq, o1, sq.size)
    oracle.orc.orc_p32_sqrt_n(sq, o2, sq.size)
    assert np.array_equal(o1, o2)


def test_from_double_matches_oracle(hc):
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-1, 1, 100_000), 10.0 ** rng.uniform(-45, 45, 100_000),
                        rng.integers(0, 2**63, 100_000, dtype=np.int64).view(np.float64),
                        [0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1e308]])
    o1 = np.empty(x.size, np.uint32)
    hc.hc_from_double_n(x, o1, x.size)
    assert np.array_equal(o1, oracle.from_double(x))


def test_decoded_mac_matches_oracle(hc):
    rng = np.random.default_rng(3)
    n = 300_000
    c, t, a = _mix(rng, n), _mix(rng, n), _mix(rng, n)
    # near-cancelling accumulators
    prod = np.empty_like(t)
    oracle.orc.orc_p32_mul_n(t, a, prod, t.size)
    sel = rng.integers(0, 9, c.size) == 0
    c[sel] = ((0 - prod[sel].astype(np.int64) + rng.integers(-3, 4, sel.sum())) & 0xFFFFFFFF).astype(np.uint32)
    out = np.empty_like(c)
    fast = hc.hc_dmac_n(c, t, a, out, c.size)
    want = np.empty_like(c)
    oracle.orc.orc_p32_add_n(c, prod, want, c.size)
    assert np.array_equal(out, want)
    assert fast > 0.5 * c.size


def test_decoded_chains_match_oracle(hc):
    rng = np.random.default_rng(4)
    nch, ln = 400, 500
    c0 = oracle.from_double(rng.uniform(-1, 1, nch))
    t = oracle.from_double(-rng.uniform(-1, 1, nch * ln))
    a = oracle.from_double(rng.uniform(-1, 1, nch * ln))
    out = np.empty(nch, np.uint32)
    hc.hc_chain(c0, t, a, out, nch, ln)
    want = c0.copy()
    for l in range(ln):
        p = np.empty(nch, np.uint32)
        oracle.orc.orc_p32_mul_n(np.ascontiguousarray(t[l::ln]), np.ascontiguousarray(a[l::ln]), p, nch)
        oracle.orc.orc_p32_add_n(want, p, want, nch)
    assert np.array_equal(out, want)


def test_chain_multiply_add_step_matches_oracle(hc):
    """The triangular-solve chain step c + t*a (computed regime entries, exact fallback)
    equals p32_add(c, p32_mul(t, a)) on random, wide-range, long-regime, cancelling and
    special operands."""
    rng = np.random.default_rng(5)
    c, t, a = _mix(rng, 40_000), _mix(rng, 40_000), _mix(rng, 40_000)
    a[::7] = oracle.P32_ONE
    c[::7] = (0 - t[::7].astype(np.uint64)).astype(np.uint32)  # c - t*1 == 0: exact cancellation
    out = np.empty_like(c)
    hc.hc_dmac_chain_n(c, t, a, out, c.size)
    p = np.empty_like(c)
    oracle.orc.orc_p32_mul_n(t, a, p, c.size)
    want = np.empty_like(c)
    oracle.orc.orc_p32_add_n(c, p, want, c.size)
    assert np.array_equal(out, want)


def test_lower_transposed_solve_matches_oracle(hc):
    """trsm_chain.cuh's L^T solve, run on the host, against the oracle's Rtrsm('L', 'L',
    'T', 'N') on Cholesky-like and wide-range triangles, with zeros and a NaR."""
    rng = np.random.default_rng(6)
    for m, kind in ((1, "u"), (9, "u"), (120, "u"), (64, "w"), (50, "nar")):
        L = oracle.from_double(rng.uniform(-1, 1, m * m))
        if kind == "w":
            L = oracle.from_double(np.sign(rng.uniform(-1, 1, m * m)) * 10.0 ** rng.uniform(-20, 20, m * m))
        for i in range(m):
            L[i + i * m] = oracle.p32(1.0 + rng.uniform(0, 1))
        b = oracle.from_double(rng.uniform(-1, 1, m))
        b[::5] = 0
        if kind == "nar":
            L[(m - 1) + 3 * m] = oracle.P32_NAR
        want = b.copy()
        oracle.orc.orc_rtrsm(b"L", b"L", b"T", b"N", m, 1, oracle.P32_ONE, L, m, want, m)
        for solve in (hc.hc_llt_solve, hc.hc_llt_solve_split):
            got = b.copy()
            solve(L, m, got, m)
            assert np.array_equal(got, want), (m, kind, solve.__name__)
        for E in (1, 4):
            got = b.copy()
            hc.hc_llt_solve_scan(L, m, got, m, E, np.zeros(2, np.int64))
            assert np.array_equal(got, want), (m, kind, "scan", E)


def test_upper_transposed_solve_matches_oracle(hc):
    """The same chain run forwards on an upper triangle (trsm_chain.cuh's llt_chain with
    upper = true) against the oracle's Rtrsm('L', 'U', 'T', 'N' / 'U'), Rtrsm.cpp:160-173."""
    rng = np.random.default_rng(16)
    for m, kind in ((1, "u"), (9, "u"), (120, "u"), (64, "w"), (50, "nar")):
        U = oracle.from_double(rng.uniform(-1, 1, m * m))
        if kind == "w":
            U = oracle.from_double(np.sign(rng.uniform(-1, 1, m * m)) * 10.0 ** rng.uniform(-20, 20, m * m))
        for i in range(m):
            U[i + i * m] = oracle.p32(1.0 + rng.uniform(0, 1))
        b = oracle.from_double(rng.uniform(-1, 1, m))
        b[::5] = 0
        if kind == "nar":
            U[2 + (m - 1) * m] = oracle.P32_NAR
        for diag, unit in ((b"N", 0), (b"U", 1)):
            want = b.copy()
            oracle.orc.orc_rtrsm(b"L", b"U", b"T", diag, m, 1, oracle.P32_ONE, U, m, want, m)
            got = b.copy()
            hc.hc_utt_solve(U, m, got, m, unit)
            assert np.array_equal(got, want), (m, kind, diag)


def test_branch_free_decode_matches_decode(hc):
    """The chain's select-only decode equals the GEMM decode on every pattern class:
    random, all regime lengths (each power of two and its neighbours), zero, extremes."""
    rng = np.random.default_rng(8)
    pw = np.array([1 << i for i in range(31)], dtype=np.uint64)
    edges = np.concatenate([pw, pw - 1, pw + 1, 0x80000000 - pw, 0x80000000 + pw, 0xFFFFFFFF - pw + 1]) % (1 << 32)
    u = np.concatenate([_mix(rng, 100_000), edges.astype(np.uint32),
                        np.array([0, 1, 0x7FFFFFFF, 0x80000001, 0xFFFFFFFF, 0x40000000, 0xC0000000], np.uint32)])
    assert hc.hc_decode_bf_mismatch(np.ascontiguousarray(u), u.size) == 0


def test_chain_of_additions_matches_oracle(hc):
    """chain_add_run (blocks without a branch, failed blocks replayed exactly) equals the
    reference's p32_add applied in order, on runs that cancel, go wide and hit zero."""
    rng = np.random.default_rng(12)
    for trial in range(300):
        n = int(rng.integers(0, 70))
        kind = trial % 3
        if kind == 0:
            q = oracle.from_double(rng.uniform(-1, 1, n))
        elif kind == 1:
            q = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 10.0 ** rng.uniform(-40, 40, n))
        else:  # values that cancel the running sum exactly now and then
            q = oracle.from_double(rng.choice([-1.0, 1.0, 0.5, -0.5, 0.0, 3.0, -3.0], n))
        c0 = int(oracle.from_double(np.array([rng.uniform(-2, 2)]))[0])
        want = np.array([c0], np.uint32)
        for k in range(n):
            oracle.orc.orc_p32_add_n(want, q[k:k + 1].copy(), want, 1)
        assert hc.hc_chain_add(c0, np.ascontiguousarray(q), n) == int(want[0]), (trial, n)


def test_fp64_chain_step_matches_oracle_across_binade_gaps(hc):
    """The FP64 step of the triangular-solve chain (add in FP64, round to the posit's
    fraction width with a magic constant, hand risky steps to the exact path) equals
    p32_add for operand gaps of 0..40 binades -- the exact, the risky (25..30) and the
    absorbed (> 30) ranges -- near-ties, cancellations, zeros and the regime extremes."""
    rng = np.random.default_rng(21)
    n = 300_000
    base = rng.uniform(-30, 30, n)
    gap = rng.integers(0, 41, n)
    t = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 2.0 ** base * rng.uniform(1, 2, n))
    q = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 2.0 ** (base - gap) * rng.uniform(1, 2, n))
    # near-ties: q just around half an ulp of t (t's last fraction bits flipped by q)
    tie = oracle.to_double(t[:50_000])
    q[:50_000] = oracle.from_double(tie * 2.0 ** -28 * rng.choice([1.0, -1.0, 0.999999, 1.000001], 50_000))
    q[50_000:60_000] = (0 - t[50_000:60_000].astype(np.uint64)).astype(np.uint32)  # exact cancellation
    q[60_000:62_000] = 0
    t[62_000:64_000] = oracle.from_double(np.sign(rng.uniform(-1, 1, 2000)) * 2.0 ** rng.uniform(95, 118, 2000))
    out = np.empty_like(t)
    flagged = hc.hc_f64_add_n(t, q, out, n)
    want = np.empty_like(t)
    oracle.orc.orc_p32_add_n(t, q, want, n)
    assert np.array_equal(out, want)
    assert 0 < flagged < n // 2  # near-ties sit in the risky 25..30-binade band by design


def _oracle_mac(c, t, a):
    p = np.empty_like(c)
    oracle.orc.orc_p32_mul_n(t, a, p, c.size)
    out = np.empty_like(c)
    oracle.orc.orc_p32_add_n(c, p, out, c.size)
    return out


@pytest.mark.parametrize("use_table", [1, 0])
def test_fp64_multiply_add_matches_oracle(hc, use_table):
    """The FP64 form of c + t*a (the GEMM inner step: the product rounded once by an FMA
    onto the posit grid, the sum rounded by a magic constant) equals
    p32_add(c, p32_mul(t, a)) on random, wide-range, long-regime, special and cancelling
    operands, on binade gaps across the risky band, and on products whose FP64 rounding
    lands exactly on a posit tie."""
    rng = np.random.default_rng(31)
    c, t, a = _mix(rng, 60_000), _mix(rng, 60_000), _mix(rng, 60_000)
    a[::9] = oracle.P32_ONE
    c[::9] = (0 - t[::9].astype(np.uint64)).astype(np.uint32)  # c + t*1 == 0
    out = np.empty_like(c)
    hc.hc_f64_mac_n(c, t, a, out, c.size, use_table)
    assert np.array_equal(out, _oracle_mac(c, t, a))
    # binade gaps 0..40 between the accumulator and the product
    n = 200_000
    base, gap = rng.uniform(-30, 30, n), rng.integers(0, 41, n)
    c = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 2.0 ** base * rng.uniform(1, 2, n))
    t = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 2.0 ** (base - gap) * rng.uniform(1, 2, n))
    a = oracle.from_double(rng.uniform(1, 2, n) * np.sign(rng.uniform(-1, 1, n)))
    out = np.empty_like(c)
    hc.hc_f64_mac_n(c, t, a, out, n, use_table)
    assert np.array_equal(out, _oracle_mac(c, t, a))
    # U[-1,1] data, the GEMM's usual diet: almost never leaves the FP64 path
    c, t, a = (oracle.from_double(rng.uniform(-1, 1, 200_000)) for _ in range(3))
    out = np.empty_like(c)
    flagged = hc.hc_f64_mac_n(c, t, a, out, c.size, use_table)
    assert np.array_equal(out, _oracle_mac(c, t, a))
    assert flagged < c.size // 1000
    # products whose FP64 rounding sits exactly on a posit tie (the exact product does not)
    tt, aa = np.zeros(64, np.uint32), np.zeros(64, np.uint32)
    found = hc.hc_find_tie_products(12345, 400_000_000, tt, aa, 64)
    assert found >= 4
    tt, aa = tt[:found], aa[:found]
    for cval in (0.0, 1e-9, -3.0, 1e9):
        cc = oracle.from_double(np.full(found, cval))
        out = np.empty_like(cc)
        hc.hc_f64_mac_n(cc, tt, aa, out, found, use_table)
        assert np.array_equal(out, _oracle_mac(cc, tt, aa))


@pytest.mark.parametrize("kind", ["uniform", "wide", "cancel", "mixed"])
def test_fp64_gemm_chains_match_oracle(hc, kind):
    """Whole GEMM k-chains through the kernels' FP64 step (per-binade constants, exact
    fixups) equal the reference's p32_mul/p32_add order."""
    rng = np.random.default_rng({"uniform": 41, "wide": 42, "cancel": 43, "mixed": 44}[kind])
    nch, ln = 300, 400
    if kind == "uniform":
        c0 = oracle.from_double(rng.uniform(-1, 1, nch))
        t = oracle.from_double(rng.uniform(-1, 1, nch * ln))
        a = oracle.from_double(rng.uniform(-1, 1, nch * ln))
    elif kind == "wide":
        c0 = oracle.from_double(np.sign(rng.uniform(-1, 1, nch)) * 10.0 ** rng.uniform(-20, 20, nch))
        t = oracle.from_double(np.sign(rng.uniform(-1, 1, nch * ln)) * 10.0 ** rng.uniform(-20, 20, nch * ln))
        a = oracle.from_double(np.sign(rng.uniform(-1, 1, nch * ln)) * 10.0 ** rng.uniform(-20, 20, nch * ln))
    elif kind == "cancel":
        c0 = oracle.from_double(rng.choice([1.0, -1.0, 0.5], nch))
        t = oracle.from_double(rng.choice([1.0, -1.0, 0.5, -0.5, 2.0 ** -26, -(2.0 ** -27), 0.0], nch * ln))
        a = oracle.from_double(rng.choice([1.0, -1.0, 3.0, 2.0 ** -3], nch * ln))
    else:
        c0, t, a = _mix(rng, nch // 5)[:nch], _mix(rng, nch * ln // 5), _mix(rng, nch * ln // 5)
        t, a = t[t != oracle.P32_NAR], a[a != oracle.P32_NAR]
        t, a = np.resize(t, nch * ln), np.resize(a, nch * ln)
        c0 = np.resize(c0[c0 != oracle.P32_NAR], nch)
    c0, t, a = (np.ascontiguousarray(x, dtype=np.uint32) for x in (c0, t, a))
    out = np.empty(nch, np.uint32)
    hc.hc_f64_gemm_chains(c0, t, a, out, nch, ln)
    want = c0.copy()
    for l in range(ln):
        p = np.empty(nch, np.uint32)
        oracle.orc.orc_p32_mul_n(np.ascontiguousarray(t[l::ln]), np.ascontiguousarray(a[l::ln]), p, nch)
        oracle.orc.orc_p32_add_n(want, p, want, nch)
    assert np.array_equal(out, want)



def test_scan_form_of_the_chain_matches_sequential_additions(hc):
    """The scan form of a chain of additions (step maps M -> M + c[M & 1] on the posit grid
    of the running value's binade, composed over a warp's window, cut at the first step the
    form does not cover, short windows followed by sequential runs), and the chain with
    the rounding constant's fraction width held fixed over blocks, equal chain_add_run -- itself pinned to p32_add above -- on chains that stay in one binade, drift across binades,
    cancel to zero, hit ties (halves of the grid spacing), span 80 decades, carry addends
    25..30 binades down, and wander across the scales 2^(4j) where the fraction width
    changes (2^-8, 2^-4, 2^4) or stays (1)."""
    rng = np.random.default_rng(31)
    stats = np.zeros(2, np.int64)
    for trial in range(1400):
        n = int(rng.integers(0, 1500))
        kind = trial % 7
        if kind == 6:  # a running value around 2^(4j), steps of about 1/100 of it
            s4 = 2.0 ** (4 * int(rng.integers(-2, 2)))
            q = oracle.from_double(rng.uniform(-1, 1, n) * 0.02 * s4)
            c0 = int(oracle.from_double(np.array([s4 * rng.uniform(0.9, 1.1)]))[0])
            E = int(rng.choice([1, 4, 16]))
            assert hc.hc_scan_row_check(c0, np.ascontiguousarray(q), n, E, stats) == 1, (trial, kind, n, E)
            assert hc.hc_chain_reg_check(c0, np.ascontiguousarray(q), n) == 1, (trial, kind, n, "reg")
            continue
        if kind == 0:
            q = oracle.from_double(rng.uniform(-1, 1, n) * 0.01)
        elif kind == 1:
            q = oracle.from_double(np.sign(rng.uniform(-1, 1, n)) * 10.0 ** rng.uniform(-40, 40, n))
        elif kind == 2:
            q = oracle.from_double(rng.choice([-1.0, 1.0, 0.5, -0.5, 0.0, 3.0, -3.0, 2**-20, -2**-27], n))
        elif kind == 3:
            q = oracle.from_double(rng.uniform(-1, 1, n) * 2.0 ** rng.integers(-30, 2, n))
        elif kind == 4:  # halves and quarters of the spacing near 1: ties on both parities
            q = oracle.from_double(rng.choice([-1, 1], n) * 2.0 ** -rng.integers(26, 30, n))
        else:  # addends 24..31 binades below a running value near 1
            q = oracle.from_double(rng.choice([-1, 1], n) * 2.0 ** -rng.integers(24, 32, n) * rng.uniform(1, 2, n))
        c0 = int(oracle.from_double(np.array([rng.uniform(-2, 2)]))[0])
        E = int(rng.choice([1, 2, 4, 8, 16]))  # 16: a 512-term window, as four warps of 32 lanes x 4 scan
        assert hc.hc_scan_row_check(c0, np.ascontiguousarray(q), n, E, stats) == 1, (trial, kind, n, E)
        assert hc.hc_chain_reg_check(c0, np.ascontiguousarray(q), n) == 1, (trial, kind, n, "reg")
    assert stats[0] > 0 and stats[1] > 0  # both scans and exact steps were exercised


def test_split_rounding_is_nearest_even_at_every_width(hc):
    """Veltkamp's split in FP64 (the fixed-width chain step's rounding: the high part of
    (2^sh+1)s) equals rounding the significand to 53 - sh bits, nearest, ties to even, for
    every shift the posit fraction widths need, on exact ties and their neighbours."""
    hc.hc_split_round_check.restype = ctypes.c_long
    hc.hc_split_round_check.argtypes = [ctypes.c_uint64, ctypes.c_long]
    assert hc.hc_split_round_check(20261204, 200_000) == 0


def _panel_cases(rng):
    for M, jb in ((1, 1), (5, 3), (40, 16), (300, 24), (130, 64)):
        yield "random", M, jb, oracle.from_double(rng.uniform(-1, 1, M * jb))
    for M, jb in ((64, 16), (200, 24)):  # few distinct magnitudes: equal keys, first row wins
        yield "ties", M, jb, oracle.from_double(rng.choice([-1.0, 1.0, 0.5, -0.5, 2.0], M * jb))
    A = oracle.from_double(rng.uniform(-1, 1, 100 * 16)).reshape(100, 16, order="F")
    A[:, 5] = 0  # a zero column: zero pivot, no interchange needed
    A[30, :] = 0
    yield "zero column", 100, 16, np.ascontiguousarray(A.reshape(-1, order="F"))
    for M in (80, 1000):  # NaR on the diagonal over zeros: a zero pivot below row 0
        A = oracle.from_double(rng.uniform(-1, 1, M * 16)).reshape(M, 16, order="F")
        A[:, 0] = 0
        A[0, 0] = oracle.P32_NAR
        yield "NaR over zeros", M, 16, np.ascontiguousarray(A.reshape(-1, order="F"))
    A = oracle.from_double(rng.uniform(-1, 1, 90 * 8)).reshape(90, 8, order="F")
    A[:, 3] = oracle.P32_NAR  # an all-NaR column: a NaR pivot (element-wise division)
    yield "NaR column", 90, 8, np.ascontiguousarray(A.reshape(-1, order="F"))
    A = oracle.from_double(rng.uniform(-1, 1, 120 * 12) * 1e-12).reshape(120, 12, order="F")
    yield "tiny", 120, 12, np.ascontiguousarray(A.reshape(-1, order="F"))


def test_cluster_lu_panel_restated_matches_the_reference_recursion(hc):
    """The cluster LU panel's algorithm (rows kept in place, interchanges as relabelling,
    the first-max pivot over logical rows, a zero pivot below the diagonal trading the two
    rows' column back, the FP64 steps with the table of rounding constants) equals the
    reference's recursive Rgetrf2 (the oracle) bit for bit, pivots and info included, on
    random, tie-heavy, singular, NaR and tiny panels."""
    hc.hc_lu_panel_relabel.restype = ctypes.c_int
    hc.hc_lu_panel_relabel.argtypes = [np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS"),
                                       ctypes.c_int, ctypes.c_int,
                                       np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")]
    rng = np.random.default_rng(77)
    for name, M, jb, A in _panel_cases(rng):
        g, o = A.copy(), A.copy()
        pg_, po = np.zeros(jb, np.int32), np.zeros(jb, np.int32)
        info_g = hc.hc_lu_panel_relabel(g, M, jb, pg_)
        info_o = oracle.orc.orc_rgetrf2(M, jb, o, M, po)
        assert info_g == info_o, name
        assert np.array_equal(pg_, po), name
        assert np.array_equal(g, o), name


def test_cluster_cholesky_panel_restated_matches_the_reference(hc):
    """The cluster Cholesky panel's algorithm (the holder of row k forms l_kk and 1/l_kk,
    the column below scaled by the FP64 product step, the rows updated up to the diagonal
    block's edge) equals the first jb columns of the reference's blocked Rpotrf('L') at
    nb = jb (the oracle) bit for bit on SPD panels, and gives the same info where a leading
    minor fails."""
    hc.hc_chol_panel.restype = ctypes.c_int
    hc.hc_chol_panel.argtypes = [np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS"),
                                 ctypes.c_int, ctypes.c_int]
    rng = np.random.default_rng(78)
    for M, jb, bad in ((1, 1, -1), (16, 16, -1), (100, 16, -1), (300, 24, -1), (257, 64, -1),
                       (200, 32, 20), (60, 16, 0)):
        X = rng.uniform(-1, 1, (M, M))
        S = oracle.from_double((X @ X.T / M + np.eye(M)).reshape(-1, order="F")).reshape(M, M, order="F")
        if bad >= 0:
            S[bad, bad] = oracle.p32(-1.0)
        S = np.ascontiguousarray(S.reshape(-1, order="F"))
        full = S.copy()
        info_o = oracle.orc.orc_rpotrf(b"L", M, full, M, jb)
        panel = np.ascontiguousarray(S.reshape(M, M, order="F")[:, :jb].reshape(-1, order="F"))
        info_g = hc.hc_chol_panel(panel, M, jb)
        if bad >= 0:
            assert info_g == info_o == bad + 1, (M, jb)
            continue
        want = np.ascontiguousarray(full.reshape(M, M, order="F")[:, :jb].reshape(-1, order="F"))
        assert info_g == info_o == 0
        assert np.array_equal(panel, want), (M, jb)


def test_exact_encode_round_trips_every_pattern_class(hc):
    """p32_from_double_exact (field assembly without rounding, for values that are posits)
    inverts p32_to_double on random patterns, every regime length and its neighbours,
    zero, NaR and the extremes."""
    rng = np.random.default_rng(41)
    pw = np.array([1 << i for i in range(31)], dtype=np.uint64)
    edges = np.concatenate([pw, pw - 1, pw + 1, 0x80000000 - pw, 0x80000000 + pw, 0xFFFFFFFF - pw + 1]) % (1 << 32)
    u = np.concatenate([rng.integers(0, 2**32, 2_000_000, dtype=np.uint64).astype(np.uint32), _mix(rng, 100_000),
                        edges.astype(np.uint32),
                        np.array([0, 1, 0x7FFFFFFF, 0x80000000, 0x80000001, 0xFFFFFFFF, 0x40000000], np.uint32)])
    assert hc.hc_from_double_exact_mismatch(np.ascontiguousarray(u), u.size) == 0

