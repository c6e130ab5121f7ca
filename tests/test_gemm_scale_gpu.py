"""Parity of the CUDA posit32 Rgemm at the sizes of the "Rgemm at scale" configuration,
against the reference's own compiled CPU Rgemm (oracle/_ref; the restatement where that
was not built), bit for bit (Rgemm.cpp:163-247):

* the benchmark's own problem, 8192^3 NN, alpha = -1, beta = 1, U[-1,1], generated by the
  same seeded device generator the benchmark uses: all rows of columns {0..15,
  4096..4111, 8176..8191} (first, middle and last column and row tiles);
* 4096^3 in all four transpose cases, the same column sample;
* 2048^3: the whole of C for NN, the column sample for NT / TN / TT;
* the wide-dynamic-range variant (magnitudes 10^U(-20,20), random signs) at 2048^3,
  all four transpose cases, sampled -- long regimes, many steps on the exact path;
* the LU trailing-update shapes m = n = 8192 - b, k = b, b in {16, 32, 64, 128, 256},
  sampled.

Operands are generated on the device and copied back, so the GPU and the checker see
the same patterns.  Each case runs one GEMM on the GPU and compares the sampled columns."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

M1, ONE = oracle.P32_MINUS_ONE, oracle.P32_ONE
TRANS = [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")]


def _sample_cols(n, w=16):
    if n <= 3 * w:
        return [(0, n)]
    mid = (n // 2) // w * w
    return [(0, w), (mid, mid + w), (n - w, n)]


def _run_and_check(m, n, k, ta, tb, alpha, beta, seed, dist="uniform", cols=None):
    import torch

    import posit_gpu_b200 as pg
    from posit_gpu_b200 import workloads
    A, lda, B, ldb, C, ldc = workloads.gemm_operands(m, n, k, ta, tb, seed=seed, dist=dist)
    hA = A.cpu().numpy().view(np.uint32)
    hB = B.cpu().numpy().view(np.uint32)
    hC = C.cpu().numpy().view(np.uint32)
    pg.Rgemm_dev(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    torch.cuda.synchronize()
    assert pg.device_error(True) == 0
    got = C.cpu().numpy().view(np.uint32)
    del A, B, C
    for j0, j1 in (cols if cols is not None else _sample_cols(n)):
        want, kind = oracle.rgemm_cols_checked(ta, tb, m, n, k, alpha, hA, lda, hB, ldb, beta, hC, ldc, j0, j1)
        g = got[j0 * ldc:j1 * ldc]
        bad = np.flatnonzero(g != want)
        assert bad.size == 0, (f"{ta}{tb} {m}x{n}x{k} {dist}: {bad.size} of {g.size} entries in columns "
                               f"{j0}..{j1 - 1} differ from the {kind} Rgemm (first at row {bad[0] % ldc}, "
                               f"column {j0 + bad[0] // ldc})")


def test_bench_problem_8192_nn_sampled(cuda_ok):
    """The benchmark's exact problem (workloads.GEMM_SEED, rank 0)."""
    from posit_gpu_b200 import workloads
    _run_and_check(8192, 8192, 8192, "N", "N", M1, ONE, workloads.GEMM_SEED)


@pytest.mark.parametrize("ta,tb", TRANS)
def test_4096_sampled(cuda_ok, ta, tb):
    _run_and_check(4096, 4096, 4096, ta, tb, M1, ONE, 4096 + ord(ta) * 3 + ord(tb))


def test_2048_nn_full(cuda_ok):
    _run_and_check(2048, 2048, 2048, "N", "N", M1, ONE, 2048, cols=[(j, j + 256) for j in range(0, 2048, 256)])


@pytest.mark.parametrize("ta,tb", TRANS[1:])
def test_2048_sampled(cuda_ok, ta, tb):
    _run_and_check(2048, 2048, 2048, ta, tb, M1, ONE, 2048 + ord(ta) * 3 + ord(tb))


@pytest.mark.parametrize("ta,tb", TRANS)
def test_2048_wide_range_sampled(cuda_ok, ta, tb):
    _run_and_check(2048, 2048, 2048, ta, tb, M1, ONE, 777 + ord(ta) * 3 + ord(tb), dist="wide")


@pytest.mark.parametrize("b", [16, 32, 64, 128, 256])
def test_lu_trailing_shapes_sampled(cuda_ok, b):
    m = 8192 - b
    _run_and_check(m, m, b, "N", "N", M1, ONE, 9000 + b)
