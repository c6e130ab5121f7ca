"""Batched GEMM (one persistent, graph-captured launch over a queue of output tiles):
every C must equal the oracle (the CPU Rgemm order) bit for bit, for every tile shape."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
ONE, M1, NAR = oracle.P32_ONE, oracle.P32_MINUS_ONE, oracle.P32_NAR


def _make(rng, count, max_dim=200, specials=False):
    probs = []
    for _ in range(count):
        m, n, k = (int(np.exp(rng.uniform(np.log(1), np.log(max_dim)))) for _ in range(3))
        ta, tb = rng.choice(["N", "T"]), rng.choice(["N", "T"])
        ar, ac = (m, k) if ta == "N" else (k, m)
        br, bc = (k, n) if tb == "N" else (n, k)
        A = oracle.from_double(rng.uniform(-1, 1, ar * ac))
        B = oracle.from_double(rng.uniform(-1, 1, br * bc))
        C = oracle.from_double(rng.uniform(-1, 1, m * n))
        alpha, beta = M1, ONE
        if specials:
            alpha = [ONE, M1, 0, oracle.p32(0.3), NAR][rng.integers(0, 5)]
            beta = [0, ONE, oracle.p32(-0.5), NAR][rng.integers(0, 4)]
            if rng.integers(0, 6) == 0:
                A[rng.integers(0, max(1, A.size))] = 0
        probs.append((ta, tb, m, n, k, alpha, A, max(1, ar), B, max(1, br), beta, C, max(1, m)))
    return probs


def _run(probs, table=None):
    import torch

    import posit_gpu_b200 as pg
    dev = torch.device("cuda")
    t = []
    for (ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc) in probs:
        t.append((ta, tb, m, n, k, al, torch.from_numpy(A.view(np.int32)).to(dev), lda,
                  torch.from_numpy(B.view(np.int32)).to(dev), ldb, be, torch.from_numpy(C.view(np.int32)).to(dev),
                  ldc))
    plan = pg.BatchGemmPlan(t, tile_table=table)
    plan.launch()
    torch.cuda.synchronize()
    return [x[11].cpu().numpy().view(np.uint32) for x in t]


@pytest.mark.parametrize("table", [None, [0] * 9, [1] * 9, [2] * 9])
def test_batch_gemm_bit_exact(cuda_ok, table):
    rng = np.random.default_rng(77 if table is None else 78 + table[0])
    probs = _make(rng, 60)
    outs = _run(probs, table)
    for p, got in zip(probs, outs):
        ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc = p
        want = C.copy()
        oracle.rgemm(ta, tb, m, n, k, al, A, lda, B, ldb, be, want, ldc)
        assert np.array_equal(got, want), (ta, tb, m, n, k)


def test_batch_gemm_special_values(cuda_ok):
    rng = np.random.default_rng(99)
    probs = _make(rng, 80, max_dim=90, specials=True)
    probs.append(("N", "N", 0, 5, 5, ONE, np.zeros(1, np.uint32), 1, np.zeros(25, np.uint32), 5, 0,
                  np.zeros(1, np.uint32), 1))
    outs = _run(probs)
    for p, got in zip(probs, outs):
        ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc = p
        want = C.copy()
        oracle.rgemm(ta, tb, m, n, k, al, A, lda, B, ldb, be, want, ldc)
        assert np.array_equal(got, want), (ta, tb, m, n, k, hex(al), hex(be))


def test_batch_gemm_rejects_bad_arguments(cuda_ok):
    import torch

    import posit_gpu_b200 as pg
    t = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="parameter number  8"):
        pg.BatchGemmPlan([("N", "N", 4, 4, 4, ONE, t, 4, t, 4, 0, t, 4), ("N", "N", 4, 2, 2, ONE, t, 3, t, 2, 0, t, 4)])


def test_batch_gemm_k0_every_alpha_beta(cuda_ok):
    """k = 0 in the batched kernel: TN/TT form alpha*0 and combine it with beta*C
    (Rgemm.cpp:190-203, 232-245), NaR for alpha = NaR; NN/NT only scale C."""
    rng = np.random.default_rng(123)
    probs = []
    for ta in ("N", "T"):
        for tb in ("N", "T"):
            for alpha in (0, ONE, M1, oracle.p32(0.3), NAR):
                for beta in (0, ONE, oracle.p32(0.5), NAR):
                    m, n = int(rng.integers(1, 70)), int(rng.integers(1, 70))
                    C = oracle.from_double(rng.uniform(-1, 1, m * n))
                    C[0] = NAR
                    z = np.zeros(max(1, m * n), np.uint32)
                    probs.append((ta, tb, m, n, 0, alpha, z, max(1, m), z.copy(), max(1, n), beta, C, m))
    outs = _run(probs)
    for p, got in zip(probs, outs):
        ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc = p
        want = C.copy()
        oracle.rgemm(ta, tb, m, n, k, al, A, lda, B, ldb, be, want, ldc)
        if oracle.ref is not None:
            w2 = C.copy()
            oracle.ref.ref_rgemm(ta.encode(), tb.encode(), m, n, k, al, A, lda, B, ldb, be, w2, ldc)
            assert np.array_equal(w2, want)
        assert np.array_equal(got, want), (ta, tb, m, n, hex(al), hex(be))
