"""Batched factor-and-solve (one persistent, graph-captured launch): every factor, pivot
vector, info and solution must equal the per-call path and the oracle bit for bit."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _problem(rng, kind, n, nrhs):
    if kind == 0:
        A = oracle.from_double(rng.uniform(-1, 1, n * n))
    else:
        M = rng.uniform(-1, 1, (n, n))
        A = oracle.from_double((M @ M.T / max(n, 1) + np.eye(n)).reshape(-1, order="F"))
    B = oracle.from_double(rng.uniform(-1, 1, n * nrhs))
    return A, B


def _oracle_solve(kind, n, nrhs, A, B):
    F, X = A.copy(), B.copy()
    ipiv = np.zeros(max(n, 1), np.int32)
    if kind == 0:
        info = oracle.orc.orc_rgetrf(n, n, F, max(n, 1), ipiv, 64)
        oracle.orc.orc_rgetrs(b"N", n, nrhs, F, max(n, 1), ipiv, X, max(n, 1))
    else:
        info = oracle.orc.orc_rpotrf(b"L", n, F, max(n, 1), 64)
        if info == 0:
            oracle.orc.orc_rpotrs(b"L", n, nrhs, F, max(n, 1), X, max(n, 1))
    return F, X, ipiv[:n], info


def test_batch_matches_oracle_and_per_call(cuda_ok):
    import torch

    import posit_gpu_b200 as pg
    rng = np.random.default_rng(2025)
    specs = []
    for n in (1, 2, 5, 8, 17, 31, 64, 100, 130, 257, 300):
        for kind in (0, 1):
            specs.append((kind, n, int(rng.integers(1, 5))))
    # a singular LU, a non-positive-definite Cholesky, and an LU whose first column is NaR
    # over zeros (a zero pivot below the diagonal: rows 0 and 1 trade places in every
    # column but the first)
    specs += [(0, 40, 2), (1, 45, 1), (0, 40, 2)]
    host = [_problem(rng, k, n, r) for (k, n, r) in specs]
    A0 = host[-3][0].reshape(40, 40, order="F")
    A0[:, 7] = 0
    host[-3] = (np.ascontiguousarray(A0.reshape(-1, order="F")), host[-3][1])
    S0 = host[-2][0].reshape(45, 45, order="F")
    S0[30, 30] = oracle.p32(-2.0)
    host[-2] = (np.ascontiguousarray(S0.reshape(-1, order="F")), host[-2][1])
    A1 = host[-1][0].reshape(40, 40, order="F")
    A1[:, 0] = 0
    A1[0, 0] = oracle.P32_NAR
    host[-1] = (np.ascontiguousarray(A1.reshape(-1, order="F")), host[-1][1])
    dev = torch.device("cuda")
    tens = []
    for (kind, n, r), (A, B) in zip(specs, host):
        tens.append((kind, torch.from_numpy(A.view(np.int32)).to(dev), torch.from_numpy(B.view(np.int32)).to(dev),
                     torch.zeros(max(n, 1), dtype=torch.int32, device=dev),
                     torch.zeros(1, dtype=torch.int32, device=dev)))
    plan = pg.BatchPlan(tens)
    plan.launch()
    torch.cuda.synchronize()
    for (kind, n, r), (A, B), (_, dA, dB, dp, di) in zip(specs, host, tens):
        F, X, ipiv, info = _oracle_solve(kind, n, r, A, B)
        assert int(di.item()) == info, (kind, n)
        if kind == 1 and info != 0:
            continue  # a stopped Cholesky leaves the rest of A unspecified (only info is defined)
        assert np.array_equal(dA.cpu().numpy().view(np.uint32), F), (kind, n)
        if kind == 0:
            assert np.array_equal(dp.cpu().numpy()[:n], ipiv), (kind, n)
        if info == 0:
            assert np.array_equal(dB.cpu().numpy().view(np.uint32), X), (kind, n)
    # per-call path on a few of the same problems gives the same bits
    for idx in (5, 12, 19):
        kind, n, r = specs[idx]
        A, B = host[idx]
        dA = torch.from_numpy(A.view(np.int32)).to(dev)
        dB = torch.from_numpy(B.view(np.int32)).to(dev)
        info = torch.zeros(1, dtype=torch.int32, device=dev)
        if kind == 0:
            ip = torch.zeros(n, dtype=torch.int32, device=dev)
            pg.Rgetrf_dev(n, n, dA, n, ip, info)
            pg.Rgetrs_dev("N", n, r, dA, n, ip, dB, n)
        else:
            pg.Rpotrf_dev("L", n, dA, n, info)
            pg.Rpotrs_dev("L", n, r, dA, n, dB, n)
        torch.cuda.synchronize()
        assert torch.equal(dA, tens[idx][1]) and torch.equal(dB, tens[idx][2])


def test_batch_replay_is_repeatable(cuda_ok):
    """The captured graph can be replayed (fresh inputs each time)."""
    import torch

    import posit_gpu_b200 as pg
    rng = np.random.default_rng(1)
    dev = torch.device("cuda")
    A, B = _problem(rng, 0, 50, 2)
    dA = torch.from_numpy(A.view(np.int32)).to(dev)
    dB = torch.from_numpy(B.view(np.int32)).to(dev)
    ip = torch.zeros(50, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    plan = pg.BatchPlan([(0, dA, dB, ip, info)])
    results = []
    for _ in range(3):
        dA.copy_(torch.from_numpy(A.view(np.int32)))
        dB.copy_(torch.from_numpy(B.view(np.int32)))
        plan.launch()
        torch.cuda.synchronize()
        results.append((dA.clone(), dB.clone()))
    assert all(torch.equal(results[0][0], r[0]) and torch.equal(results[0][1], r[1]) for r in results)
