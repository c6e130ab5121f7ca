/*
 * ref_glue.cpp -- plain-C entry points into the reference's own libRpack CPU
 * routines (compiled out of tree against softposit_cpp.h in this folder), plus the
 * two definitions that build needs from outside those sources:
 *   abs(posit32)  the reference's util.cpp:12-17 (util.cpp itself also drags in
 *                 LAPACK generators, so it is not compiled)
 *   iMlaenv       replaced so the block size of Rgetrf/Rpotrf is the caller's
 *                 (the reference hard-codes 64: iMlaenv.cpp:145-150, 223-228)
 * Test infrastructure only (oracle/_ref).
 */
#include <mpblas.h>
#include <mplapack.h>

posit32 abs(posit32 x)
{
    posit32 t = x;
    if (t < 0.0)
        t = -t;
    return t;
}

static int g_ref_nb = 64;

INTEGER iMlaenv(INTEGER const, const char *, const char *, INTEGER const, INTEGER const,
                INTEGER const, INTEGER const)
{
    return g_ref_nb;
}

static inline posit32 P(uint32_t u) { return posit32::bits(u); }
static inline posit32 *PP(uint32_t *u) { return reinterpret_cast<posit32 *>(u); }
static inline posit32 *PPc(const uint32_t *u) { return reinterpret_cast<posit32 *>(const_cast<uint32_t *>(u)); }

extern "C" {

void ref_set_nb(int nb) { g_ref_nb = nb; }

void ref_rgemm(char ta, char tb, int m, int n, int k, uint32_t alpha, const uint32_t *a, int lda,
               const uint32_t *b, int ldb, uint32_t beta, uint32_t *c, int ldc)
{
    char sa[2] = {ta, 0}, sb[2] = {tb, 0};
    Rgemm(sa, sb, m, n, k, P(alpha), PPc(a), lda, PPc(b), ldb, P(beta), PP(c), ldc);
}

void ref_rsyrk(char uplo, char trans, int n, int k, uint32_t alpha, const uint32_t *a, int lda,
               uint32_t beta, uint32_t *c, int ldc)
{
    char su[2] = {uplo, 0}, st[2] = {trans, 0};
    Rsyrk(su, st, n, k, P(alpha), PPc(a), lda, P(beta), PP(c), ldc);
}

void ref_rtrsm(char side, char uplo, char trans, char diag, int m, int n, uint32_t alpha,
               const uint32_t *a, int lda, uint32_t *b, int ldb)
{
    char s1[2] = {side, 0}, s2[2] = {uplo, 0}, s3[2] = {trans, 0}, s4[2] = {diag, 0};
    Rtrsm(s1, s2, s3, s4, m, n, P(alpha), PPc(a), lda, PP(b), ldb);
}

void ref_rgemv(char trans, int m, int n, uint32_t alpha, const uint32_t *a, int lda,
               const uint32_t *x, int incx, uint32_t beta, uint32_t *y, int incy)
{
    char st[2] = {trans, 0};
    Rgemv(st, m, n, P(alpha), PPc(a), lda, PPc(x), incx, P(beta), PP(y), incy);
}

int ref_iramax(int n, const uint32_t *x, int incx) { return iRamax(n, PPc(x), incx); }

void ref_rscal(int n, uint32_t da, uint32_t *x, int incx) { Rscal(n, P(da), PP(x), incx); }

void ref_rlaswp(int n, uint32_t *a, int lda, int k1, int k2, int *ipiv, int incx)
{
    Rlaswp(n, PP(a), lda, k1, k2, ipiv, incx);
}

int ref_rgetrf2(int m, int n, uint32_t *a, int lda, int *ipiv)
{
    INTEGER info = 0;
    Rgetrf2(m, n, PP(a), lda, ipiv, info);
    return info;
}

int ref_rgetrf(int m, int n, uint32_t *a, int lda, int *ipiv, int nb)
{
    INTEGER info = 0;
    g_ref_nb = nb;
    Rgetrf(m, n, PP(a), lda, ipiv, info);
    return info;
}

int ref_rgetrs(char trans, int n, int nrhs, const uint32_t *a, int lda, int *ipiv, uint32_t *b, int ldb)
{
    INTEGER info = 0;
    char st[2] = {trans, 0};
    Rgetrs(st, n, nrhs, PPc(a), lda, ipiv, PP(b), ldb, info);
    return info;
}

int ref_rpotrf2(char uplo, int n, uint32_t *a, int lda)
{
    INTEGER info = 0;
    char su[2] = {uplo, 0};
    Rpotrf2(su, n, PP(a), lda, info);
    return info;
}

int ref_rpotrf(char uplo, int n, uint32_t *a, int lda, int nb)
{
    INTEGER info = 0;
    char su[2] = {uplo, 0};
    g_ref_nb = nb;
    Rpotrf(su, n, PP(a), lda, info);
    return info;
}

int ref_rpotrs(char uplo, int n, int nrhs, const uint32_t *a, int lda, uint32_t *b, int ldb)
{
    INTEGER info = 0;
    char su[2] = {uplo, 0};
    Rpotrs(su, n, nrhs, PPc(a), lda, PP(b), ldb, info);
    return info;
}

}
