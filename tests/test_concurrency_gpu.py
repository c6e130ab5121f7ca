"""Device factorizations and solves in flight at once on separate streams -- as the serving
loop runs them -- give the bits of the same calls run one after another."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _mat(rng, kind, n):
    if kind == 0:
        return oracle.from_double(rng.uniform(-1, 1, n * n))
    M = rng.uniform(-1, 1, (n, n))
    return oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))


@pytest.mark.parametrize("mix", ["lu", "cholesky", "both"])
def test_concurrent_factor_and_solve_match_sequential(cuda_ok, mix):
    import torch

    import posit_gpu_b200 as pg
    dev = torch.device("cuda")
    rng = np.random.default_rng({"lu": 1, "cholesky": 2, "both": 3}[mix])
    count, nrhs = 48, 4
    sizes = [int(x) for x in np.rint(np.exp(rng.uniform(np.log(300), np.log(3000), count)))]
    kinds = [0] * count if mix == "lu" else [1] * count if mix == "cholesky" else \
        [int(k) for k in rng.integers(0, 2, count)]
    mats = [torch.from_numpy(_mat(rng, k, n).view(np.int32)).to(dev) for k, n in zip(kinds, sizes)]
    rhs = [torch.from_numpy(oracle.from_double(rng.uniform(-1, 1, n * nrhs)).view(np.int32)).to(dev)
           for n in sizes]

    def fresh():
        bufs = [(A.clone(), B.clone(), torch.zeros(n, dtype=torch.int32, device=dev),
                 torch.zeros(1, dtype=torch.int32, device=dev)) for A, B, n in zip(mats, rhs, sizes)]
        torch.cuda.synchronize()  # made on the default stream, used on others
        return bufs

    def run(bufs, kind, n, st):
        A, B, ipiv, info = bufs
        if kind == 0:
            pg.Rgetrf_dev(n, n, A, n, ipiv, info, nb=64, stream=st)
            pg.Rgetrs_dev("N", n, nrhs, A, n, ipiv, B, n, stream=st)
        else:
            pg.Rpotrf_dev("L", n, A, n, info, nb=64, stream=st)
            pg.Rpotrs_dev("L", n, nrhs, A, n, B, n, stream=st)

    seq = fresh()
    for b, k, n in zip(seq, kinds, sizes):
        run(b, k, n, None)
        torch.cuda.synchronize()
    for rep in range(3):
        outs = fresh()
        streams = [torch.cuda.Stream() for _ in sizes]
        for b, k, n, st in zip(outs, kinds, sizes, streams):
            run(b, k, n, st)
        torch.cuda.synchronize()
        assert pg.device_error(True) == 0
        bad = [(i, kinds[i], sizes[i]) for i in range(count)
               if not all(torch.equal(x, y) for x, y in zip(outs[i], seq[i]))]
        assert not bad, (mix, rep, bad)
