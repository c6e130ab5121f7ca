"""posit_rgemm_dev_noalloc: the GEMM entry point for callers that cannot allocate device
memory (their memory manager owns the GPU's memory, or cudaMalloc/cudaFree would
synchronise the device in a loop that must not stall).  Its scratch is a static 64 MiB
device array inside the library, shared by every call on the device.

Checked through the C ABI against the ordinary device entry point, posit_rgemm_dev,
and against the oracle, bit for bit (the tolerance every GEMM test here uses), on two
calls in a row with different shapes and transposes -- the second call must not see
anything the first one left in the shared array (a NaR in the first call's operands must
not leak into the second's NaR flags).  Argument errors keep their Rgemm info codes, and
calls that need no scratch are not refused.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _lib():
    import posit_gpu_b200 as pg
    return pg._lib


def _dev(x):
    import torch
    return torch.from_numpy(x.view(np.int32)).cuda()


def _case(rng, ta, tb, m, n, k):
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    A = oracle.from_double(rng.uniform(-1, 1, ar * ac))
    B = oracle.from_double(rng.uniform(-1, 1, br * bc))
    C = oracle.from_double(rng.uniform(-1, 1, m * n))
    return A, ar, B, br, C


def _call(fn, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, extra):
    return fn(ta.encode(), tb.encode(), m, n, k, alpha, ctypes.c_void_p(A.data_ptr()), lda,
              ctypes.c_void_p(B.data_ptr()), ldb, beta, ctypes.c_void_p(C.data_ptr()), ldc, *extra)


def test_noalloc_matches_device_entry_point_twice(cuda_ok):
    import torch
    lib = _lib()
    rng = np.random.default_rng(2024)
    alpha, beta = oracle.P32_MINUS_ONE, oracle.p32(0.75)
    # two calls in a row, different shapes/transposes; the second is smaller than the first
    for call, (ta, tb, m, n, k) in enumerate((("N", "N", 300, 260, 1000), ("T", "N", 130, 70, 90))):
        A, lda, B, ldb, C = _case(rng, ta, tb, m, n, k)
        if call == 0:  # NaR in row 5 of op(A) and column 3 of op(B): flags the second call must not see
            A[5] = oracle.P32_NAR
            B[3 * ldb] = oracle.P32_NAR
        dA, dB = _dev(A), _dev(B)
        c_ref, c_new = _dev(C), _dev(C)
        rc = _call(lib.posit_rgemm_dev, ta, tb, m, n, k, alpha, dA, lda, dB, ldb, beta, c_ref, m,
                   (None, 0, None))
        assert rc == 0
        rc = _call(lib.posit_rgemm_dev_noalloc, ta, tb, m, n, k, alpha, dA, lda, dB, ldb, beta, c_new, m,
                   (None,))
        assert rc == 0
        torch.cuda.synchronize()
        assert torch.equal(c_ref, c_new), f"{ta}{tb} {m}x{n}x{k}"
        want = C.copy()
        assert oracle.rgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, want, m) == 0
        assert np.array_equal(c_new.cpu().numpy().view(np.uint32), want), f"{ta}{tb} vs oracle"
        assert lib.posit_device_error(1) == 0


def test_noalloc_refuses_shapes_beyond_its_scratch(cuda_ok):
    import torch
    lib = _lib()
    limit = 64 << 20
    m = n = k = 4096  # needs 256 MiB of scratch
    assert lib.posit_rgemm_workspace_size(b"N", b"N", m, n, k) > limit
    t = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = _call(lib.posit_rgemm_dev_noalloc, "N", "N", m, n, k, oracle.P32_ONE, t, m, t, k, 0, t, m, (None,))
    assert rc == -6
    assert b"static" in lib.posit_strerror(rc)
    assert int(t.abs().sum()) == 0  # nothing was launched


def test_noalloc_argument_errors_and_calls_without_scratch(cuda_ok):
    """A bad argument returns its Rgemm info code even for a shape beyond the scratch;
    alpha == 0 and k == 0 form no product, need no scratch and run at any size."""
    import torch
    lib = _lib()
    t = torch.zeros(16, dtype=torch.int32, device="cuda")
    big = 4096
    assert _call(lib.posit_rgemm_dev_noalloc, "X", "N", big, big, big, oracle.P32_ONE, t, big, t, big, 0, t, big,
                 (None,)) == 1
    assert _call(lib.posit_rgemm_dev_noalloc, "N", "N", big, big, big, oracle.P32_ONE, t, big - 1, t, big, 0, t,
                 big, (None,)) == 8
    # alpha == 0, beta == 0 at 4096^3: C <- 0 without scratch
    C = torch.full((big * big,), 0x40000000, dtype=torch.int32, device="cuda")
    assert _call(lib.posit_rgemm_dev_noalloc, "N", "N", big, big, big, 0, t, big, t, big, 0, C, big, (None,)) == 0
    torch.cuda.synchronize()
    assert int((C != 0).sum()) == 0
    # k == 0, TN, alpha == NaR: alpha*0 is NaR everywhere (Rgemm.cpp:193-201)
    assert _call(lib.posit_rgemm_dev_noalloc, "T", "N", big, big, 0, oracle.P32_NAR, t, 1, t, 1, oracle.p32(0.5), C,
                 big, (None,)) == 0
    torch.cuda.synchronize()
    assert bool((C == -2**31).all())
