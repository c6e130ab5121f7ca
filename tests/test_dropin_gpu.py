"""The drop-in check: the reference's OWN GPU-accelerated factorizations
(libRpack/Rgetrf_opencl.cpp, Rgetrf2_opencl.cpp, Rpotrf_opencl.cpp), compiled unchanged,
call RgemmG for their trailing updates; linked against the B200 RgemmG
(posit_gpu_b200/integration/Rgemm_b200.cpp) they must reproduce the reference's CPU
Rgetrf / Rpotrf bit for bit at the same block size.  (With the reference's OpenCL
kernels they could not: those accumulate NN/NT products in a different order.)"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(cuda_ok):
    lib = oracle.load_ref_dropin()
    if lib is None or oracle.ref is None:
        pytest.skip("oracle/_ref drop-in library not built (needs the reference tree at build time)")
    return lib


@pytest.mark.parametrize("n,nb", [(200, 32), (300, 64), (640, 128)])
def test_reference_rgetrf_opencl_with_b200_rgemmg(dropin, n, nb):
    rng = np.random.default_rng(n + nb)
    A = oracle.from_double(rng.uniform(-1, 1, n * n))
    gpu, cpu = A.copy(), A.copy()
    pg_, pc = np.zeros(n, np.int32), np.zeros(n, np.int32)
    info_g = dropin.refd_rgetrf_opencl(n, n, gpu, n, pg_, nb)
    info_c = oracle.ref.ref_rgetrf(n, n, cpu, n, pc, nb)
    assert info_g == info_c == 0
    assert np.array_equal(pg_, pc)
    assert np.array_equal(gpu, cpu)


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n,nb", [(200, 32), (520, 64)])
def test_reference_rpotrf_opencl_with_b200_rgemmg(dropin, uplo, n, nb):
    rng = np.random.default_rng(7 * n + nb)
    M = rng.uniform(-1, 1, (n, n))
    S = oracle.from_double((M @ M.T / n + np.eye(n)).reshape(-1, order="F"))
    gpu, cpu = S.copy(), S.copy()
    info_g = dropin.refd_rpotrf_opencl(uplo.encode(), n, gpu, n, nb)
    info_c = oracle.ref.ref_rpotrf(uplo.encode(), n, cpu, n, nb)
    assert info_g == info_c == 0
    assert np.array_equal(gpu, cpu)
