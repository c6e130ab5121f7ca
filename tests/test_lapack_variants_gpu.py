"""The device variants beyond LU and lower Cholesky, bit for bit against the reference's
own compiled CPU routines (oracle/_ref) and the restatement:

* Rpotrf('U') -- left-looking, blocked by nb, each upper entry updated by dot products
  over the rows above it (Rpotrf.cpp:96-118, Rpotrf2.cpp:86-131, Rsyrk.cpp:182-195,
  Rtrsm.cpp:160-173): its bits depend on nb, so it is compared at the same nb, including
  nb = 1 and nb >= n (Rpotrf2 on the whole matrix);
* Rpotrs('U') -- U^T forward, then U backward (Rpotrs.cpp:84-95);
* Rgetrs('T') and ('C') -- U^T forward, L^T backward (unit), interchanges in reverse
  (Rgetrs.cpp:99-113)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _ge(rng, m, n, kind="u"):
    if kind == "wide":
        x = np.sign(rng.uniform(-1, 1, m * n)) * 10.0 ** rng.uniform(-20, 20, m * n)
        return oracle.from_double(x)
    return oracle.from_double(rng.uniform(-1, 1, m * n))


def _spd(rng, n):
    M = rng.uniform(-1, 1, (n, n))
    return oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))


def _ref_rpotrf_upper(S, n, nb):
    """Upper Cholesky by the reference's own code where built, and the restatement."""
    o = S.copy()
    info_o = oracle.orc.orc_rpotrf(b"U", n, o, n, nb)
    if oracle.ref is not None:
        r = S.copy()
        oracle.ref.ref_set_nb(nb)
        info_r = oracle.ref.ref_rpotrf(b"U", n, r, n, nb)
        assert info_r == info_o and np.array_equal(r, o), "restatement and reference disagree"
    return o, info_o


@pytest.mark.parametrize("n,nb", [(1, 64), (5, 2), (64, 16), (129, 1), (200, 64), (200, 300), (300, 256),
                                  (520, 64), (520, 256), (1024, 64), (1024, 256)])
def test_rpotrf_upper_bit_exact(cuda_ok, n, nb):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(7 * n + nb)
    S = _spd(rng, n)
    want, info_o = _ref_rpotrf_upper(S, n, nb)
    g = S.copy()
    info_g = pg.Rpotrf("U", n, g, n, nb)
    assert info_g == info_o == 0
    bad = np.flatnonzero(g != want)
    assert bad.size == 0, f"{bad.size} entries differ (first at row {bad[0] % n}, column {bad[0] // n})"


def test_rpotrf_upper_default_nb_is_the_references(cuda_ok):
    """nb <= 0 on the device path is 64, the block size the reference's Rpotrf takes from
    iMlaenv."""
    import torch

    import posit_gpu_b200 as pg
    n = 333
    rng = np.random.default_rng(333)
    S = _spd(rng, n)
    want, _ = _ref_rpotrf_upper(S, n, 64)
    dA = torch.from_numpy(S.view(np.int32).copy()).cuda()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    pg.Rpotrf_dev("U", n, dA, n, info)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    assert np.array_equal(dA.cpu().numpy().view(np.uint32), want)


def test_rpotrf_upper_not_positive_definite(cuda_ok):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(19)
    n = 150
    S = _spd(rng, n).reshape(n, n, order="F")
    S[90, 90] = oracle.p32(-1.0)
    S = np.ascontiguousarray(S.reshape(-1, order="F"))
    for nb in (16, 64, 200):
        g = S.copy()
        _, info_o = _ref_rpotrf_upper(S, n, nb)
        assert pg.Rpotrf("U", n, g, n, nb) == info_o > 0


@pytest.mark.parametrize("n,nrhs", [(1, 1), (9, 2), (200, 4), (700, 16), (3000, 2)])
def test_rpotrs_upper_bit_exact(cuda_ok, n, nrhs):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(13 * n + nrhs)
    S = _spd(rng, n)
    assert oracle.orc.orc_rpotrf(b"U", n, S, n, 64) == 0
    B = _ge(rng, n, nrhs)
    g, o = B.copy(), B.copy()
    pg.Rpotrs("U", n, nrhs, S, n, g, n)
    oracle.orc.orc_rpotrs(b"U", n, nrhs, S, n, o, n)
    if oracle.ref is not None:
        r = B.copy()
        oracle.ref.ref_rpotrs(b"U", n, nrhs, S, n, r, n)
        assert np.array_equal(r, o)
    assert np.array_equal(g, o)


@pytest.mark.parametrize("trans", ["T", "C"])
@pytest.mark.parametrize("n,nrhs,kind", [(1, 1, "u"), (7, 3, "u"), (150, 5, "u"), (513, 16, "u"),
                                         (300, 3, "wide"), (2500, 2, "u")])
def test_rgetrs_transposed_bit_exact(cuda_ok, trans, n, nrhs, kind):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(n + 31 * nrhs)
    A = _ge(rng, n, n, kind)
    ipiv = np.zeros(n, np.int32)
    oracle.orc.orc_rgetrf(n, n, A, n, ipiv, 64)
    B = _ge(rng, n, nrhs, kind)
    g, o = B.copy(), B.copy()
    pg.Rgetrs(trans, n, nrhs, A, n, ipiv, g, n)
    oracle.orc.orc_rgetrs(trans.encode(), n, nrhs, A, n, ipiv, o, n)
    if oracle.ref is not None:
        r = B.copy()
        oracle.ref.ref_rgetrs(trans.encode(), n, nrhs, A, n, ipiv, r, n)
        assert np.array_equal(r, o)
    assert np.array_equal(g, o)
