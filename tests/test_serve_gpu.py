"""Served solves: every solution and info equals the per-call path bit for bit, served
alone and in a concurrent mix, through the factor cache and after evictions; admission,
cancellation and bad arguments behave as include/posit_gpu.h declares."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _problem(rng, kind, n):
    if kind == 0:
        return oracle.from_double(rng.uniform(-1, 1, n * n))
    M = rng.uniform(-1, 1, (n, n))
    return oracle.from_double((M @ M.T / max(n, 1) + np.eye(n)).reshape(-1, order="F"))


def _rhs(rng, n, nrhs):
    return oracle.from_double(rng.uniform(-1, 1, n * nrhs))


def _per_call(pg, kind, n, nrhs, A, B):
    """The plain drop-in path: Rgetrf + Rgetrs (Rpotrf + Rpotrs) on host buffers."""
    F, X = A.copy(), B.copy()
    if kind == 0:
        ipiv = np.zeros(max(n, 1), np.int32)
        info = pg.Rgetrf(n, n, F, max(n, 1), ipiv, nb=64)
        pg.Rgetrs("N", n, nrhs, F, max(n, 1), ipiv, X, max(n, 1))
    else:
        info = pg.Rpotrf("L", n, F, max(n, 1), nb=64)
        if info == 0:
            pg.Rpotrs("L", n, nrhs, F, max(n, 1), X, max(n, 1))
    return X, info


def _workload(seed=11):
    """Matrices on both sides of the batched/blocked split (batch_max_n = 96 below), a
    singular LU and a non-positive-definite Cholesky, and ~30% repeat requests that reuse
    an earlier matrix with new right-hand sides."""
    rng = np.random.default_rng(seed)
    mats = []
    for n in (1, 3, 16, 40, 90, 96, 97, 150, 300, 520):
        for kind in (0, 1):
            mats.append((kind, n, _problem(rng, kind, n)))
    # singular LU (n = 150: blocked path) and indefinite Cholesky (n = 40: batched path)
    i_lu = [i for i, m in enumerate(mats) if m[0] == 0 and m[1] == 150][0]
    A = mats[i_lu][2].reshape(150, 150, order="F").copy()
    A[:, 33] = 0
    mats[i_lu] = (0, 150, np.ascontiguousarray(A.reshape(-1, order="F")))
    i_ch = [i for i, m in enumerate(mats) if m[0] == 1 and m[1] == 40][0]
    S = mats[i_ch][2].reshape(40, 40, order="F").copy()
    S[20, 20] = oracle.p32(-3.0)
    mats[i_ch] = (1, 40, np.ascontiguousarray(S.reshape(-1, order="F")))
    reqs = [(mid, int(rng.integers(1, 5))) for mid in range(len(mats))]
    for _ in range(9):  # repeats, each after its matrix's first request
        mid = int(rng.integers(0, len(mats)))
        first = [i for i, (m, _) in enumerate(reqs) if m == mid][0]
        reqs.insert(int(rng.integers(first + 1, len(reqs) + 1)), (mid, int(rng.integers(1, 5))))
    out = [(mid, nrhs, _rhs(rng, mats[mid][1], nrhs)) for mid, nrhs in reqs]
    return mats, out, (i_lu, i_ch)


def _pinned(torch, a):
    t = torch.from_numpy(a.view(np.int32)).pin_memory()
    return t


def test_served_alone_and_in_a_mix_match_per_call(cuda_ok):
    import torch

    import posit_gpu_b200 as pg
    mats, reqs, (i_lu, i_ch) = _workload()
    want = []
    for mid, nrhs, B in reqs:
        kind, n, A = mats[mid]
        want.append(_per_call(pg, kind, n, nrhs, A, B))

    # alone: one request at a time
    alone = []
    with pg.Server(batch_max_n=96) as srv:
        first = set()
        for mid, nrhs, B in reqs:
            kind, n, A = mats[mid]
            X = np.zeros_like(B)
            res = srv.wait(srv.submit(kind, n, nrhs, A, B, X, matrix_id=mid))
            assert res["status"] == 0, res
            assert res["cache_hit"] == (mid in first)
            assert res["path"] == (0 if n <= 96 else 1)
            first.add(mid)
            alone.append((X, res["info"]))
        st = srv.stats()
        assert st["cache_hits"] == len(reqs) - len(mats)
        assert st["failed"] == 0 and st["completed"] == len(reqs)

    # mix: everything submitted at once; half the buffers page-locked, half pageable
    mixed = []
    with pg.Server(batch_max_n=96, lanes=6) as srv:
        tickets, outs = [], []
        for i, (mid, nrhs, B) in enumerate(reqs):
            kind, n, A = mats[mid]
            if i % 2:
                Ab, Bb, Xb = _pinned(torch, A), _pinned(torch, B), _pinned(torch, np.zeros_like(B))
            else:
                Ab, Bb, Xb = A, B, np.zeros_like(B)
            tickets.append(srv.submit(kind, n, nrhs, Ab, Bb, Xb, matrix_id=mid))
            outs.append(Xb)
        for t, Xb in zip(tickets, outs):
            res = srv.wait(t)
            assert res["status"] == 0, res
            X = Xb.numpy().view(np.uint32) if hasattr(Xb, "numpy") else Xb
            mixed.append((X, res["info"]))
        assert srv.stats()["inflight_peak"] > 1

    for (mid, nrhs, B), (Xw, iw), (Xa, ia), (Xm, im) in zip(reqs, want, alone, mixed):
        kind, n, _ = mats[mid]
        assert iw == ia == im, (kind, n)
        if iw == 0:
            assert np.array_equal(Xa, Xw), (kind, n)
            assert np.array_equal(Xm, Xw), (kind, n)
    info_of = {mid: iw for (mid, _, _), (_, iw) in zip(reqs, want)}
    assert info_of[i_lu] > 0 and info_of[i_ch] > 0


def test_served_small_problems_match_oracle(cuda_ok):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(3)
    with pg.Server() as srv:
        for kind in (0, 1):
            for n in (1, 7, 33):
                A, B = _problem(rng, kind, n), _rhs(rng, n, 2)
                X = np.zeros_like(B)
                res = srv.wait(srv.submit(kind, n, 2, A, B, X))
                F, Xo = A.copy(), B.copy()
                ipiv = np.zeros(n, np.int32)
                if kind == 0:
                    info = oracle.orc.orc_rgetrf(n, n, F, n, ipiv, 64)
                    oracle.orc.orc_rgetrs(b"N", n, 2, F, n, ipiv, Xo, n)
                else:
                    info = oracle.orc.orc_rpotrf(b"L", n, F, n, 64)
                    oracle.orc.orc_rpotrs(b"L", n, 2, F, n, Xo, n)
                assert res["status"] == 0 and res["info"] == info == 0
                assert np.array_equal(X, Xo), (kind, n)


def test_budget_evicts_least_recently_used_factors(cuda_ok):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(5)
    n = 200  # batched path: factor block ~160 KB
    mats = [_problem(rng, i % 2, n) for i in range(10)]
    with pg.Server(memory_budget=1 << 20) as srv:
        for i, A in enumerate(mats):
            B = _rhs(rng, n, 1)
            X = np.zeros_like(B)
            res = srv.wait(srv.submit(i % 2, n, 1, A, B, X, matrix_id=i))
            Xw, iw = _per_call(pg, i % 2, n, 1, A, B)
            assert res["status"] == 0 and res["info"] == iw == 0 and not res["cache_hit"]
            assert np.array_equal(X, Xw)
            st = srv.stats()
            assert st["bytes_peak"] <= st["budget_bytes"] == 1 << 20
        assert srv.stats()["evictions"] > 0
        B = _rhs(rng, n, 3)
        # the oldest factor was evicted: a request without A cannot be served
        res = srv.wait(srv.submit(0, n, 3, None, B, np.zeros_like(B), matrix_id=0))
        assert res["status"] == pg.E_NOT_CACHED
        # the newest is still cached: solve only, same bits as factor + solve
        X = np.zeros_like(B)
        res = srv.wait(srv.submit(1, n, 3, None, B, X, matrix_id=9))
        assert res["status"] == 0 and res["cache_hit"]
        assert np.array_equal(X, _per_call(pg, 1, n, 3, mats[9], B)[0])
        # a cached id with another kind or order is refused
        res = srv.wait(srv.submit(0, n, 1, mats[9], B[:n], np.zeros(n, np.uint32), matrix_id=9))
        assert res["status"] == pg.E_MISMATCH


def test_cancel_bad_arguments_and_shutdown(cuda_ok):
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(9)
    srv = pg.Server(max_inflight=1, lanes=1, memory_budget=256 << 20)
    with pytest.raises(ValueError):
        srv.submit(5, 4, 1, np.zeros(16, np.uint32), np.zeros(4, np.uint32), np.zeros(4, np.uint32))
    with pytest.raises(ValueError):
        srv.submit(0, 4, 1, None, np.zeros(4, np.uint32), np.zeros(4, np.uint32))  # no A, no id
    with pytest.raises(pg.PositError, match="out of device memory"):
        big = np.zeros(1, np.uint32)
        srv.submit(0, 9000, 1, big, big, big)  # 324 MB matrix > 256 MB budget
    A = _problem(rng, 0, 1200)
    B = _rhs(rng, 1200, 1)
    X0 = np.zeros_like(B)
    t0 = srv.submit(0, 1200, 1, A, B, X0)
    small = [(_problem(rng, 1, 20), _rhs(rng, 20, 1)) for _ in range(4)]
    outs = [np.zeros(20, np.uint32) for _ in small]
    ts = [srv.submit(1, 20, 1, a, b, x) for (a, b), x in zip(small, outs)]
    cancelled = srv.cancel(ts[-1])
    assert srv.wait(t0)["status"] == 0
    assert np.array_equal(X0, _per_call(pg, 0, 1200, 1, A, B)[0])
    for t, (a, b), x in zip(ts[:-1], small[:-1], outs[:-1]):
        assert srv.wait(t)["status"] == 0
        assert np.array_equal(x, _per_call(pg, 1, 20, 1, a, b)[0])
    last = srv.wait(ts[-1])
    assert last["status"] == (pg.E_CANCELLED if cancelled else 0)
    with pytest.raises(pg.PositError):
        srv.wait(ts[-1])  # taken already
    # shutdown with work queued: returns, and queued requests are cancelled
    for _ in range(3):
        srv.submit(0, 300, 2, _problem(rng, 0, 300), _rhs(rng, 300, 2), np.zeros(600, np.uint32))
    srv.close()


def test_burst_admits_largest_work_first(cuda_ok):
    """Requests submitted within one order window are admitted largest work first: behind a
    request that holds the only slot, four more of different n are admitted by decreasing
    n, whatever their submission order, and each result still equals the per-call one."""
    import posit_gpu_b200 as pg
    rng = np.random.default_rng(21)
    with pg.Server(max_inflight=1, lanes=2, batch_max_n=64, order_window_ms=60000) as srv:
        A0, B0 = _problem(rng, 0, 1500), _rhs(rng, 1500, 1)
        t0 = srv.submit(0, 1500, 1, A0, B0, np.zeros_like(B0))
        sizes = [300, 900, 400, 600]
        probs = [(_problem(rng, 0, n), _rhs(rng, n, 1)) for n in sizes]
        outs = [np.zeros_like(b) for _, b in probs]
        ts = [srv.submit(0, n, 1, a, b, x) for n, (a, b), x in zip(sizes, probs, outs)]
        assert srv.wait(t0)["status"] == 0
        res = [srv.wait(t) for t in ts]
        assert all(r["status"] == 0 for r in res)
        admitted = sorted(range(4), key=lambda i: res[i]["queue_ms"])
        assert [sizes[i] for i in admitted] == [900, 600, 400, 300]
        for n, (a, b), x in zip(sizes, probs, outs):
            assert np.array_equal(x, _per_call(pg, 0, n, 1, a, b)[0])
