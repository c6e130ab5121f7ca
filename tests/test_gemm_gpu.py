"""Parity of the CUDA posit32 Rgemm (through the C ABI) against the oracle."""
import numpy as np
import pytest

import oracle
from tests import posit_data as pd

pytestmark = pytest.mark.gpu

ONE, NAR, M1 = oracle.P32_ONE, oracle.P32_NAR, oracle.P32_MINUS_ONE


def _case(rng, ta, tb, m, n, k, alpha, beta, kind="uniform", pad=0):
    ar, ac = (m, k) if ta in "nN" else (k, m)
    br, bc = (k, n) if tb in "nN" else (n, k)
    lda, ldb, ldc = max(1, ar + pad), max(1, br + pad), max(1, m + pad)
    A = pd.colmajor(rng, ar, ac, lda, kind)
    B = pd.colmajor(rng, br, bc, ldb, kind)
    C = pd.colmajor(rng, m, n, ldc, kind)
    return A, lda, B, ldb, C, ldc


def _run_both(ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc, cols=None):
    import posit_gpu_b200 as pg
    Cg = C.copy()
    pg.Rgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cg, ldc)
    Co = C.copy()
    assert oracle.rgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Co, ldc, cols=cols) == 0
    return Cg, Co


TRANS = [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")]


@pytest.mark.parametrize("ta,tb", TRANS)
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 3, 7), (33, 17, 65), (64, 64, 16), (100, 70, 49), (129, 130, 131)])
def test_small_shapes_bit_exact(cuda_ok, ta, tb, m, n, k):
    rng = np.random.default_rng(1000 + m * 7 + n * 3 + k)
    alpha, beta = oracle.p32(rng.uniform(-2, 2)), oracle.p32(rng.uniform(-2, 2))
    A, lda, B, ldb, C, ldc = _case(rng, ta, tb, m, n, k, alpha, beta, pad=3)
    Cg, Co = _run_both(ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc)
    assert np.array_equal(Cg, Co)


@pytest.mark.parametrize("ta,tb", TRANS)
@pytest.mark.parametrize("alpha,beta", [(ONE, 0), (ONE, ONE), (M1, ONE), (0, 0x20000000), (0, 0), (NAR, ONE), (ONE, NAR)])
def test_alpha_beta_special(cuda_ok, ta, tb, alpha, beta):
    rng = np.random.default_rng(7)
    m, n, k = 70, 45, 33
    A, lda, B, ldb, C, ldc = _case(rng, ta, tb, m, n, k, alpha, beta)
    Cg, Co = _run_both(ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc)
    assert np.array_equal(Cg, Co)


@pytest.mark.parametrize("ta,tb", TRANS)
def test_wide_range_and_specials(cuda_ok, ta, tb):
    rng = np.random.default_rng(11)
    m, n, k = 96, 80, 200
    alpha, beta = M1, ONE
    A, lda, B, ldb, C, ldc = _case(rng, ta, tb, m, n, k, alpha, beta, kind="wide")
    # sprinkle zeros, NaR, maxpos/minpos and exact negatives for cancellation
    for buf in (A, B, C):
        idx = rng.integers(0, buf.size, size=buf.size // 50)
        buf[idx[0::4]] = 0
        buf[idx[1::4]] = 0x7FFFFFFF
        buf[idx[2::4]] = 0x00000001
        buf[idx[3::4][:2]] = NAR
    Cg, Co = _run_both(ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc)
    assert np.array_equal(Cg, Co)


def test_config1_512_nn(cuda_ok):
    """512^3 NN, alpha=1, beta=0.5, ld=512, U[-1,1]: full bit compare."""
    rng = np.random.default_rng(20240101)
    n = 512
    A = pd.uniform(rng, (n * n,))
    B = pd.uniform(rng, (n * n,))
    C = pd.uniform(rng, (n * n,))
    alpha, beta = oracle.p32(1.0), oracle.p32(0.5)
    Cg, Co = _run_both("N", "N", n, n, n, alpha, beta, A, n, B, n, C, n)
    assert np.array_equal(Cg, Co)


@pytest.mark.parametrize("ta,tb", TRANS)
def test_2048_sampled_columns(cuda_ok, ta, tb):
    rng = np.random.default_rng(2048)
    n = 2048
    A = pd.uniform(rng, (n * n,))
    B = pd.uniform(rng, (n * n,))
    C = pd.uniform(rng, (n * n,))
    import posit_gpu_b200 as pg
    Cg = C.copy()
    pg.Rgemm(ta, tb, n, n, n, M1, A, n, B, n, ONE, Cg, n)
    for j0 in (0, 1000, n - 24):
        Co = C.copy()
        oracle.rgemm(ta, tb, n, n, n, M1, A, n, B, n, ONE, Co, n, cols=(j0, j0 + 24))
        assert np.array_equal(Cg[j0 * n:(j0 + 24) * n], Co[j0 * n:(j0 + 24) * n])


def test_only_submatrix_touched(cuda_ok):
    """Guard band: entries of C outside the m x n submatrix are never written."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(3)
    m, n, k, ldc = 37, 29, 20, 50
    A = pd.uniform(rng, (m * k,))
    B = pd.uniform(rng, (k * n,))
    C = pd.uniform(rng, (ldc * n + 64,))
    Cg = C.copy()
    pg.Rgemm("N", "N", m, n, k, M1, A, m, B, k, ONE, Cg, ldc)
    mask = np.zeros(C.size, bool)
    for j in range(n):
        mask[j * ldc:j * ldc + m] = True
    assert np.array_equal(Cg[~mask], C[~mask])


K0_ALPHAS = [0, ONE, M1, oracle.p32(0.3), NAR]
K0_BETAS = [0, ONE, oracle.p32(0.5), NAR]


def _k0_want(ta, tb, m, n, alpha, beta, C):
    """k = 0 through the restatement and, where built, the reference's own Rgemm: for
    TN/TT it still forms alpha*0 and combines it with beta*C (Rgemm.cpp:190-203,
    232-245), so alpha = NaR gives NaR."""
    z = np.zeros(max(1, m * n), np.uint32)
    want = C.copy()
    assert oracle.rgemm(ta, tb, m, n, 0, alpha, z, max(1, m), z, max(1, n), beta, want, m) == 0
    if oracle.ref is not None:
        w2 = C.copy()
        oracle.ref.ref_rgemm(ta.encode(), tb.encode(), m, n, 0, alpha, z, max(1, m), z, max(1, n), beta, w2, m)
        assert np.array_equal(w2, want), "restatement and reference disagree at k = 0"
    return want


@pytest.mark.parametrize("ta,tb", TRANS)
def test_k0_every_alpha_beta(cuda_ok, ta, tb):
    """k = 0, every (alpha, beta) of the special set, on the host, device and no-alloc
    entry points."""
    import torch

    import posit_gpu_b200 as pg
    rng = np.random.default_rng(5)
    m, n = 19, 13
    z = np.zeros(max(1, m * n), np.uint32)
    C = pd.uniform(rng, (m * n,))
    C[3], C[7] = NAR, 0
    for alpha in K0_ALPHAS:
        for beta in K0_BETAS:
            want = _k0_want(ta, tb, m, n, alpha, beta, C)
            Cg = C.copy()
            pg.Rgemm(ta, tb, m, n, 0, alpha, z, max(1, m), z, max(1, n), beta, Cg, m)
            assert np.array_equal(Cg, want), ("host", hex(alpha), hex(beta))
            dz = torch.zeros(max(1, m * n), dtype=torch.int32, device="cuda")
            for fn in (pg.Rgemm_dev, pg.Rgemm_dev_noalloc):
                dC = torch.from_numpy(C.view(np.int32).copy()).cuda()
                fn(ta, tb, m, n, 0, alpha, dz, max(1, m), dz, max(1, n), beta, dC, m)
                torch.cuda.synchronize()
                got = dC.cpu().numpy().view(np.uint32)
                assert np.array_equal(got, want), (fn.__name__, hex(alpha), hex(beta))
