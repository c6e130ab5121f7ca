"""Device-resident LU / Cholesky and solves against the oracle (the reference's operation
order) and against the reference's own outputs (golden vectors)."""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _ge(rng, m, n):
    return oracle.from_double(rng.uniform(-1, 1, m * n))


def _spd(rng, n):
    M = rng.uniform(-1, 1, (n, n))
    return oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))


@pytest.mark.parametrize("m,n,nb", [(1, 1, 256), (5, 5, 2), (37, 37, 8), (100, 100, 32), (300, 300, 64),
                                    (257, 257, 256), (700, 700, 256), (90, 60, 16), (60, 90, 16),
                                    (5000, 130, 64), (4100, 600, 512), (4500, 300, 600)])
def test_rgetrf_bit_exact(cuda_ok, m, n, nb):
    """Panels up to 4096 rows (and 512 columns) run in one thread block, taller or wider
    ones as two launches per column; both are covered."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(m * 1000 + n)
    A = _ge(rng, m, n)
    g, o = A.copy(), A.copy()
    pg_, po = np.zeros(min(m, n), np.int32), np.zeros(min(m, n), np.int32)
    info_g = pg.Rgetrf(m, n, g, m, pg_, nb)
    info_o = oracle.orc.orc_rgetrf(m, n, o, m, po, nb)
    assert info_g == info_o
    assert np.array_equal(pg_, po)
    assert np.array_equal(g, o)


def test_rgetrf_singular_and_zero_pivots(cuda_ok):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(5)
    n = 80
    A = _ge(rng, n, n).reshape(n, n, order="F")
    A[:, 10] = 0                      # exactly zero column -> zero pivot at step 10
    A[:, 40] = A[:, 3]                # dependent column
    A[17, :] = 0
    A = np.ascontiguousarray(A.reshape(-1, order="F"))
    g, o = A.copy(), A.copy()
    pg_, po = np.zeros(n, np.int32), np.zeros(n, np.int32)
    info_g = pg.Rgetrf(n, n, g, n, pg_, 16)
    info_o = oracle.orc.orc_rgetrf(n, n, o, n, po, 16)
    assert info_g == info_o > 0
    assert np.array_equal(pg_, po) and np.array_equal(g, o)


@pytest.mark.parametrize("m,n", [(80, 80), (3000, 40)])
def test_rgetrf_zero_pivot_below_a_nar_row(cuda_ok, m, n):
    """Column 0 is NaR on the diagonal and zero below: iRamax takes the first zero (row 1),
    the pivot is zero, so no interchange happens and u comes from row 0 (the NaR row);
    info is 1.  One panel CTA (m = 80) and a cluster of three (m = 3000)."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(m + 7)
    A = _ge(rng, m, n).reshape(m, n, order="F")
    A[:, 0] = 0
    A[0, 0] = oracle.P32_NAR
    A = np.ascontiguousarray(A.reshape(-1, order="F"))
    g, o = A.copy(), A.copy()
    pg_, po = np.zeros(n, np.int32), np.zeros(n, np.int32)
    info_g = pg.Rgetrf(m, n, g, m, pg_, 16)
    info_o = oracle.orc.orc_rgetrf(m, n, o, m, po, 16)
    assert info_g == info_o == 1
    assert pg_[0] == po[0] == 2
    assert np.array_equal(pg_, po) and np.array_equal(g, o)


@pytest.mark.parametrize("n,nrhs", [(1, 1), (7, 3), (150, 5), (513, 16)])
def test_rgetrs_bit_exact(cuda_ok, n, nrhs):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(n + nrhs)
    A = _ge(rng, n, n)
    ipiv = np.zeros(n, np.int32)
    assert oracle.orc.orc_rgetrf(n, n, A, n, ipiv, 64) == 0
    B = _ge(rng, n, nrhs)
    g, o = B.copy(), B.copy()
    pg.Rgetrs("N", n, nrhs, A, n, ipiv, g, n)
    oracle.orc.orc_rgetrs(b"N", n, nrhs, A, n, ipiv, o, n)
    assert np.array_equal(g, o)


@pytest.mark.parametrize("n,nb", [(1, 256), (5, 2), (64, 16), (300, 64), (520, 256), (700, 128), (900, 600),
                                  (4300, 256)])
def test_rpotrf_lower_bit_exact(cuda_ok, n, nb):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(n * 3 + nb)
    S = _spd(rng, n)
    g, o = S.copy(), S.copy()
    info_g = pg.Rpotrf("L", n, g, n, nb)
    info_o = oracle.orc.orc_rpotrf(b"L", n, o, n, nb)
    assert info_g == info_o == 0
    assert np.array_equal(g, o)


@pytest.mark.parametrize("n,bad", [(120, 77), (700, 20)])
def test_rpotrf_not_positive_definite(cuda_ok, n, bad):
    """The leading minor of order bad+1 fails: in a later one-CTA panel (n = 120) or in the
    first panel, held by a cluster of six CTAs (n = 700)."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(9)
    S = _spd(rng, n).reshape(n, n, order="F")
    S[bad, bad] = oracle.p32(-1.0)
    S = np.ascontiguousarray(S.reshape(-1, order="F"))
    g, o = S.copy(), S.copy()
    assert pg.Rpotrf("L", n, g, n, 32) == oracle.orc.orc_rpotrf(b"L", n, o, n, 32) == bad + 1


@pytest.mark.parametrize("n,nrhs", [(1, 1), (9, 2), (200, 4), (400, 16)])
def test_rpotrs_bit_exact(cuda_ok, n, nrhs):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(11 * n + nrhs)
    S = _spd(rng, n)
    assert oracle.orc.orc_rpotrf(b"L", n, S, n, 64) == 0
    B = _ge(rng, n, nrhs)
    g, o = B.copy(), B.copy()
    pg.Rpotrs("L", n, nrhs, S, n, g, n)
    oracle.orc.orc_rpotrs(b"L", n, nrhs, S, n, o, n)
    assert np.array_equal(g, o)


@pytest.mark.parametrize("n,kind", [(300, "wide"), (700, "ties"), (1500, "u"), (11600, "u")])
def test_rpotrs_any_factor_bit_exact(cuda_ok, n, kind):
    """Rpotrs on lower triangles that are no Cholesky factor: entries over 40 decades, or
    powers of two that make the running sums hit grid ties, zeros in the right-hand sides,
    a NaR in one column -- the transposed solve's chain leaves its binade, cancels and
    takes the exact path often.  n = 11600 is past the FP64 term buffers' shared-memory
    limit: the terms are kept as posit patterns."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(n)
    if kind == "wide":
        Lf = np.sign(rng.uniform(-1, 1, (n, n))) * 10.0 ** rng.uniform(-20, 20, (n, n))
    elif kind == "ties":
        Lf = rng.choice([-1, 1], (n, n)) * 2.0 ** -rng.integers(0, 30, (n, n))
    else:
        Lf = rng.uniform(-1, 1, (n, n)) / np.sqrt(n)
    Lf = np.tril(Lf)
    np.fill_diagonal(Lf, 1.0 + rng.uniform(0, 1, n))
    L = oracle.from_double(Lf.reshape(-1, order="F"))
    nrhs = 3 if n < 5000 else 1
    B = oracle.from_double(rng.uniform(-1, 1, n * nrhs))
    B[::7] = 0
    if kind == "wide":
        L[(n - 1) + 5 * n] = oracle.P32_NAR  # column 5 of L^T's row: x_5 and those above it NaR
    g, o = B.copy(), B.copy()
    pg.Rpotrs("L", n, nrhs, L, n, g, n)
    oracle.orc.orc_rpotrs(b"L", n, nrhs, L, n, o, n)
    assert np.array_equal(g, o)


def test_lapack_matches_reference_golden(cuda_ok):
    """LU, Cholesky and both solves against outputs of the reference's own code."""
    import posit_gpu_b200 as pg
    g = np.load(os.path.join(GOLD, "lapack.npz"))
    for i, (n, nb, nrhs, info, cinfo, uinfo) in enumerate(g["meta"]):
        lu = g[f"A{i}"].copy()
        ipiv = np.zeros(n, np.int32)
        assert pg.Rgetrf(n, n, lu, n, ipiv, nb) == info
        assert np.array_equal(lu, g[f"lu{i}"]) and np.array_equal(ipiv, g[f"ipiv{i}"])
        x = g[f"b{i}"].copy()
        pg.Rgetrs("N", n, nrhs, lu, n, ipiv, x, n)
        assert np.array_equal(x, g[f"x{i}"])
        ch = g[f"S{i}"].copy()
        assert pg.Rpotrf("L", n, ch, n, nb) == cinfo
        assert np.array_equal(ch, g[f"chl{i}"])
        xs = g[f"b{i}"].copy()
        pg.Rpotrs("L", n, nrhs, ch, n, xs, n)
        assert np.array_equal(xs, g[f"xs{i}"])


def test_bad_variant_letters_are_refused(cuda_ok):
    """uplo / trans outside the reference's letters return the info code of argument 1
    (Rpotrf.cpp:64-72, Rgetrs.cpp:60-71)."""
    import posit_gpu_b200 as pg
    S = np.zeros(4, np.uint32)
    with pytest.raises(ValueError):
        pg.Rpotrf("X", 2, S, 2)
    with pytest.raises(ValueError):
        pg.Rpotrs("X", 2, 1, S, 2, S.copy(), 2)
    with pytest.raises(ValueError):
        pg.Rgetrs("X", 2, 1, S, 2, np.ones(2, np.int32), S.copy(), 2)
