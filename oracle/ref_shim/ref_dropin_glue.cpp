/*
 * ref_dropin_glue.cpp -- plain-C entry points into the reference's OWN GPU-accelerated
 * factorizations, Rgetrf_opencl / Rpotrf_opencl (libRpack/Rgetrf_opencl.cpp:32-154,
 * Rgetrf2_opencl.cpp:32-193, Rpotrf_opencl.cpp:32-166), compiled unchanged and linked
 * with posit_gpu_b200/integration/Rgemm_b200.cpp, so their RgemmG trailing updates run
 * on the B200 library.  Used by the drop-in test only (oracle/_ref).
 */
#include <mpblas.h>
#include <mplapack.h>

extern "C" void ref_set_nb(int nb);

static inline posit32 *PP(uint32_t *u) { return reinterpret_cast<posit32 *>(u); }

extern "C" {

int refd_rgetrf_opencl(int m, int n, uint32_t *a, int lda, int *ipiv, int nb)
{
    INTEGER info = 0;
    Rgetrf_opencl(m, n, PP(a), lda, ipiv, info, nb);
    return info;
}

int refd_rpotrf_opencl(char uplo, int n, uint32_t *a, int lda, int nb)
{
    INTEGER info = 0;
    char su[2] = {uplo, 0};
    ref_set_nb(nb); /* Rpotrf_opencl takes its block size from iMlaenv */
    Rpotrf_opencl(su, n, PP(a), lda, info);
    return info;
}
}
