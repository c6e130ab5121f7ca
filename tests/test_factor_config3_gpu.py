"""Device-resident factorizations on the configuration-3 systems (n = 1024 and 4096,
nb = 256): factors, pivots, right-hand side and solution must hash to exactly what the
reference's own CPU Rgemv/Rgetrf/Rgetrs/Rpotrf/Rpotrs produced (tests/golden/
factor_hashes.json), and the FP64 error report of the solve is printed beside it."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "factor_hashes.json")


def _h(t):
    return hashlib.sha256(t.cpu().numpy().tobytes()).hexdigest()


def _cases():
    if not os.path.exists(GOLD):
        return []
    return sorted(json.load(open(GOLD)).values(), key=lambda c: (c["kind"], c["n"]))


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_config3_factorization_matches_reference(cuda_ok, case):
    import torch

    import posit_gpu_b200 as pg
    from posit_gpu_b200 import accuracy

    n, nb = case["n"], case["nb"]
    A_h, x_h = mg.regen_factor_inputs(case)
    assert hashlib.sha256(A_h.tobytes()).hexdigest() == case["A_sha256"], "input generator drifted"
    dev = torch.device("cuda")
    A = torch.from_numpy(A_h.view(np.int32)).to(dev)
    x = torch.from_numpy(x_h.view(np.int32)).to(dev)
    b = torch.zeros(n, dtype=torch.int32, device=dev)
    # b = A*x: the NN GEMM with one column is Rgemv 'N' with beta = 0, bit for bit
    pg.Rgemm_dev("N", "N", n, 1, n, pg.P32_ONE, A, n, x, n, 0, b, n)
    torch.cuda.synchronize()
    assert _h(b) == case["b_sha256"]
    F = A.clone()
    rhs = b.clone()
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    if case["kind"] == "lu":
        ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
        pg.Rgetrf_dev(n, n, F, n, ipiv, info, nb=nb)
        pg.Rgetrs_dev("N", n, 1, F, n, ipiv, rhs, n)
        torch.cuda.synchronize()
        assert _h(ipiv) == case["ipiv_sha256"]
    else:
        pg.Rpotrf_dev("L", n, F, n, info, nb=nb)
        pg.Rpotrs_dev("L", n, 1, F, n, rhs, n)
        torch.cuda.synchronize()
    assert int(info.item()) == case["info"]
    assert _h(F) == case["factor_sha256"]
    assert _h(rhs) == case["x_sha256"]
    rep = accuracy.solve_report(A, b, rhs, x_true=x, n=n, spd=case["kind"] == "chol")
    print(case["name"], json.dumps(rep))
    assert rep["backward_error"] < 1e-6
