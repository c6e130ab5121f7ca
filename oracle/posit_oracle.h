/*
 * posit_oracle.h -- CPU restatement of the reference's posit(32,2) arithmetic and
 * posit BLAS/LAPACK operation orders.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is linked by the
 * tests, by the smoke check and by the CPU-baseline leg of the benchmark, never by
 * the product library (posit_gpu_b200/), which must fail loudly if its CUDA code is
 * missing rather than fall back to anything here.
 *
 * Arithmetic:
 *   add / mul      restate the SoftPosit algorithm as ported in the reference,
 *                  libRpack/kernel_entry.cl:88-538, including its truncating
 *                  alignment and its sticky-bit window.  Pinned against that very
 *                  source compiled from the reference tree (oracle/_ref).
 *   sub            add(a, -b), the reference's C++ class mapping of a - b.
 *   div/sqrt/from_double
 *                  no in-tree source exists (SoftPosit is an absent third-party
 *                  dependency, no pinned version).  Written from the posit standard
 *                  as correctly rounded round-to-nearest-even on the bit pattern,
 *                  never rounding to zero or NaR.  Parity with upstream SoftPosit is
 *                  UNPINNED for these three.
 */
#ifndef POSIT_ORACLE_H
#define POSIT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_P32_NAR  0x80000000u
#define ORC_P32_ONE  0x40000000u

uint32_t orc_p32_add(uint32_t a, uint32_t b);
uint32_t orc_p32_sub(uint32_t a, uint32_t b);
uint32_t orc_p32_mul(uint32_t a, uint32_t b);
uint32_t orc_p32_div(uint32_t a, uint32_t b);
uint32_t orc_p32_sqrt(uint32_t a);
uint32_t orc_p32_neg(uint32_t a);
uint32_t orc_p32_abs(uint32_t a);
uint32_t orc_p32_from_double(double x);
double   orc_p32_to_double(uint32_t a);
/* element-wise helpers used by the Python side of the tests */
void orc_p32_add_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n);
void orc_p32_mul_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n);
void orc_p32_div_n(const uint32_t *a, const uint32_t *b, uint32_t *out, int64_t n);
void orc_p32_sqrt_n(const uint32_t *a, uint32_t *out, int64_t n);
void orc_p32_from_double_n(const double *x, uint32_t *out, int64_t n);
void orc_p32_to_double_n(const uint32_t *a, double *out, int64_t n);

/* BLAS level 3 (libRpack/Rgemm.cpp:62-251): returns 0 or the BLAS info code of
 * the first bad argument (the reference calls Mxerbla, which exits). */
int orc_rgemm(char transa, char transb, int m, int n, int k, uint32_t alpha,
              const uint32_t *a, int lda, const uint32_t *b, int ldb,
              uint32_t beta, uint32_t *c, int ldc);
/* Same, restricted to columns [j0, j1) of C (a bounded sample for timing). */
int orc_rgemm_cols(char transa, char transb, int m, int n, int k, uint32_t alpha,
                   const uint32_t *a, int lda, const uint32_t *b, int ldb,
                   uint32_t beta, uint32_t *c, int ldc, int j0, int j1);
int orc_num_threads(void);

/* BLAS/LAPACK routines on the factorization path (libRpack/R*.cpp). */
int orc_iramax(int n, const uint32_t *x, int incx);
void orc_rscal(int n, uint32_t da, uint32_t *x, int incx);
void orc_rlaswp(int n, uint32_t *a, int lda, int k1, int k2, const int *ipiv, int incx);
int orc_rtrsm(char side, char uplo, char transa, char diag, int m, int n, uint32_t alpha,
              const uint32_t *a, int lda, uint32_t *b, int ldb);
int orc_rsyrk(char uplo, char trans, int n, int k, uint32_t alpha, const uint32_t *a,
              int lda, uint32_t beta, uint32_t *c, int ldc);
int orc_rgemv(char trans, int m, int n, uint32_t alpha, const uint32_t *a, int lda,
              const uint32_t *x, int incx, uint32_t beta, uint32_t *y, int incy);
int orc_rgetrf2(int m, int n, uint32_t *a, int lda, int *ipiv);
int orc_rgetrf(int m, int n, uint32_t *a, int lda, int *ipiv, int nb);
int orc_rgetrs(char trans, int n, int nrhs, const uint32_t *a, int lda, const int *ipiv,
               uint32_t *b, int ldb);
int orc_rpotrf2(char uplo, int n, uint32_t *a, int lda);
int orc_rpotrf(char uplo, int n, uint32_t *a, int lda, int nb);
int orc_rpotrs(char uplo, int n, int nrhs, const uint32_t *a, int lda, uint32_t *b, int ldb);

#ifdef __cplusplus
}
#endif
#endif
