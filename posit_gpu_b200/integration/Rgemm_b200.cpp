// Rgemm_b200.cpp -- drop-in replacement for the reference's libRpack/Rgemm_opencl.cpp.
//
// Compile it in place of Rgemm_opencl.cpp, against the same softposit_cpp.h and
// libRpack headers, and link libposit_gpu_b200.so: libRpack's Rgetrf_opencl,
// Rgetrf2_opencl, Rpotrf_opencl and the driver programs then run their trailing-update
// GEMMs on the B200 kernels without a change to their source.
//
// Signatures as declared by the reference: RgemmG in libRpack/mpblas_posit.h:49-55,
// initOpenCL in libRpack/def.h:63.  The semantics are the CPU Rgemm's
// (libRpack/Rgemm.cpp:62-251): bit-identical results for every transpose case, 'C' is a
// transpose, illegal arguments go to Mxerbla with Rgemm's parameter numbers.
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "softposit_cpp.h"
#include "posit_gpu.h"

typedef int mplapackint;
void Mxerbla(const char *srname, int info);

static_assert(sizeof(posit32) == sizeof(uint32_t), "posit32 is one 32-bit word");

void initOpenCL(void)
{
    int rc = posit_init();
    if (rc) {
        fprintf(stderr, "initOpenCL: %s\n", posit_strerror(rc));
        exit(-1);
    }
}

void RgemmG(const char *transa, const char *transb, mplapackint const m, mplapackint const n,
            mplapackint const k, posit32 const alpha, posit32 *A, mplapackint const lda, posit32 *B,
            mplapackint const ldb, posit32 const beta, posit32 *C, mplapackint const ldc)
{
    int rc = posit_rgemm(transa[0], transb[0], m, n, k, alpha.value, reinterpret_cast<const uint32_t *>(A), lda,
                         reinterpret_cast<const uint32_t *>(B), ldb, beta.value, reinterpret_cast<uint32_t *>(C),
                         ldc);
    if (rc > 0) {
        Mxerbla("RgemmG", rc);
    } else if (rc < 0) {
        fprintf(stderr, "RgemmG: %s\n", posit_strerror(rc));
        exit(-1);
    }
}
