"""The oracle is pinned against the reference's own outputs (golden vectors made by the
reference's compiled code), and -- where oracle/_ref is built -- against that code live."""
import hashlib
import json
import os
from fractions import Fraction

import numpy as np
import pytest

import oracle
from tests.golden import make_golden as mg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _vec(f, a, b):
    out = np.empty_like(a)
    f(a, b, out, a.size)
    return out


def test_ops_match_reference_golden():
    g = np.load(os.path.join(GOLD, "ops.npz"))
    assert g["a"].size > 10000
    assert np.array_equal(_vec(oracle.orc.orc_p32_add_n, g["a"], g["b"]), g["add"])
    assert np.array_equal(_vec(oracle.orc.orc_p32_mul_n, g["a"], g["b"]), g["mul"])


def test_known_encodings():
    o = oracle.orc
    assert o.orc_p32_add(0x40000000, 0x40000000) == 0x48000000  # 1 + 1 = 2
    assert o.orc_p32_add(0x38000000, 0x38000000) == 0x40000000  # 0.5 + 0.5 = 1
    assert o.orc_p32_add(0x40000000, 0xC0000000) == 0          # 1 - 1 = 0
    assert o.orc_p32_mul(0x7FFFFFFF, 0x7FFFFFFF) == 0x7FFFFFFF  # maxpos^2 saturates
    assert o.orc_p32_mul(1, 1) == 1                            # minpos^2 saturates
    assert o.orc_p32_mul(0x80000000, 0) == 0x80000000          # NaR before zero
    assert o.orc_p32_add(0, 0x80000000) == 0x80000000
    assert oracle.p32(1.0) == 0x40000000 and oracle.p32(-1.0) == 0xC0000000


def test_rgemm_matches_reference_golden():
    g = np.load(os.path.join(GOLD, "rgemm.npz"))
    meta = g["meta"]
    for i, row in enumerate(meta):
        ta, tb, m, n, k, alpha, beta, lda, ldb, ldc = row
        C = g[f"C{i}"].copy()
        info = oracle.orc.orc_rgemm(bytes([ta]), bytes([tb]), m, n, k, alpha, g[f"A{i}"], lda, g[f"B{i}"],
                                    ldb, beta, C, ldc)
        assert info == 0
        assert np.array_equal(C, g[f"out{i}"]), f"case {i} ({chr(ta)}{chr(tb)} {m}x{n}x{k})"


def test_rgemm_hashes_match_reference():
    with open(os.path.join(GOLD, "hashes.json")) as f:
        cases = json.load(f)
    for c in cases:
        A, B, C = mg.regen_inputs(c)
        assert hashlib.sha256(A.tobytes()).hexdigest() == c["input_sha256"], "input generator drifted"
        n = c["n"]
        oracle.rgemm(c["ta"], c["tb"], n, n, n, c["alpha"], A, n, B, n, c["beta"], C, n)
        assert hashlib.sha256(C.tobytes()).hexdigest() == c["sha256"], c["name"]


def test_lapack_matches_reference_golden():
    g = np.load(os.path.join(GOLD, "lapack.npz"))
    for i, (n, nb, nrhs, info, cinfo, uinfo) in enumerate(g["meta"]):
        lu = g[f"A{i}"].copy()
        ipiv = np.zeros(n, dtype=np.int32)
        assert oracle.orc.orc_rgetrf(n, n, lu, n, ipiv, nb) == info
        assert np.array_equal(lu, g[f"lu{i}"]) and np.array_equal(ipiv, g[f"ipiv{i}"])
        x = g[f"b{i}"].copy()
        oracle.orc.orc_rgetrs(b"N", n, nrhs, lu, n, ipiv, x, n)
        assert np.array_equal(x, g[f"x{i}"])
        ch = g[f"S{i}"].copy()
        assert oracle.orc.orc_rpotrf(b"L", n, ch, n, nb) == cinfo
        assert np.array_equal(ch, g[f"chl{i}"])
        xs = g[f"b{i}"].copy()
        oracle.orc.orc_rpotrs(b"L", n, nrhs, ch, n, xs, n)
        assert np.array_equal(xs, g[f"xs{i}"])
        chu = g[f"S{i}"].copy()
        assert oracle.orc.orc_rpotrf(b"U", n, chu, n, nb) == uinfo
        assert np.array_equal(chu, g[f"chu{i}"])


@pytest.mark.skipif(oracle.ref is None, reason="oracle/_ref not built (needs the reference tree)")
def test_ops_match_reference_live():
    rng = np.random.default_rng(99)
    n = 2_000_000
    a = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    for fo, fr in ((oracle.orc.orc_p32_add_n, oracle.ref.ref_p32_add_n),
                   (oracle.orc.orc_p32_mul_n, oracle.ref.ref_p32_mul_n)):
        assert np.array_equal(_vec(fo, a, b), _vec(fr, a, b))


@pytest.mark.skipif(oracle.ref is None, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("nb", [2, 8, 32])
def test_factorizations_match_reference_live(nb):
    rng = np.random.default_rng(nb)
    n = 96
    A = oracle.from_double(rng.uniform(-1, 1, n * n))
    l1, l2 = A.copy(), A.copy()
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    assert oracle.orc.orc_rgetrf(n, n, l1, n, p1, nb) == oracle.ref.ref_rgetrf(n, n, l2, n, p2, nb)
    assert np.array_equal(l1, l2) and np.array_equal(p1, p2)
    M = rng.uniform(-1, 1, (n, n))
    S = oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))
    for uplo in (b"L", b"U"):
        c1, c2 = S.copy(), S.copy()
        assert oracle.orc.orc_rpotrf(uplo, n, c1, n, nb) == oracle.ref.ref_rpotrf(uplo, n, c2, n, nb)
        assert np.array_equal(c1, c2)


def _val(u):
    """Exact rational value of a posit32 pattern (None for NaR)."""
    u = int(u) & 0xFFFFFFFF
    if u == 0:
        return Fraction(0)
    if u == 0x80000000:
        return None
    return Fraction(oracle.orc.orc_p32_to_double(u))


def _is_nearest(q, r):
    """r is a nearest posit to the exact q (neighbours r-1, r+1 are not closer)."""
    vr = _val(r)
    for nb_ in ((r - 1) & 0xFFFFFFFF, (r + 1) & 0xFFFFFFFF):
        if nb_ in (0, 0x80000000):
            continue
        vn = _val(nb_)
        if abs(vn - q) < abs(vr - q):
            return False
    return True


def test_div_sqrt_correctly_rounded():
    """Division and square root have no in-tree reference source; check the
    restatement is correctly rounded against exact rational arithmetic."""
    rng = np.random.default_rng(5)
    o = oracle.orc
    for _ in range(1500):
        a = int(rng.integers(1, 0x7FFFFFFF))
        b = int(rng.integers(1, 0x7FFFFFFF))
        r = o.orc_p32_div(a, b)
        q = _val(a) / _val(b)
        if 2.0 ** -120 < q < 2.0 ** 120:
            assert _is_nearest(q, r), (hex(a), hex(b), hex(r))
        s = o.orc_p32_sqrt(a)
        vs = _val(s)
        lo, hi = _val((s - 1) & 0xFFFFFFFF), _val((s + 1) & 0xFFFFFFFF)
        va = _val(a)
        # sqrt(a) lies between the midpoints to both neighbours
        assert ((lo + vs) / 2) ** 2 <= va <= ((vs + hi) / 2) ** 2, hex(a)
    assert o.orc_p32_div(0x40000000, 0) == 0x80000000
    assert o.orc_p32_sqrt(0xC0000000) == 0x80000000
    assert o.orc_p32_sqrt(0x40000000) == 0x40000000


def test_column_slice_checker_matches_whole_rgemm():
    """oracle.rgemm_cols_checked (the reference's Rgemm on a slice of C's columns) equals
    the same columns of the whole restated Rgemm, for every transpose case."""
    rng = np.random.default_rng(1)
    for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
        m, n, k = 37, 29, 23
        ar = m if ta == "N" else k
        br = k if tb == "N" else n
        A = oracle.from_double(rng.uniform(-1, 1, m * k))
        B = oracle.from_double(rng.uniform(-1, 1, k * n))
        C = oracle.from_double(rng.uniform(-1, 1, m * n))
        full = C.copy()
        oracle.rgemm(ta, tb, m, n, k, oracle.P32_MINUS_ONE, A, ar, B, br, oracle.p32(0.5), full, m)
        for j0, j1 in ((0, 5), (10, 29), (28, 29)):
            got, _ = oracle.rgemm_cols_checked(ta, tb, m, n, k, oracle.P32_MINUS_ONE, A, ar, B, br,
                                               oracle.p32(0.5), C, m, j0, j1)
            assert np.array_equal(got, full[j0 * m:j1 * m]), (ta, tb, j0)
