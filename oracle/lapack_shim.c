/*
 * LAPACK/BLAS name shim for the reference oracle build (test infrastructure only).
 *
 * The reference declares the Fortran LAPACK/BLAS entry points with 64-bit
 * `long` integers (src/MatrixSolver.h:246-247, src/MatrixOperations.cpp:21-40).
 * This image has no system LAPACK; numpy ships an ILP64 OpenBLAS whose
 * exported names carry a `scipy_` prefix and a `_64_` suffix.  These
 * forwarding definitions let the unmodified reference sources link against it.
 * Character arguments get their hidden Fortran length (1) passed explicitly.
 */
#include <stddef.h>

typedef long lint;

extern void scipy_dgbtrf_64_(const lint*, const lint*, const lint*, const lint*, double*,
                             const lint*, lint*, lint*);
extern void scipy_dgbtrs_64_(const char*, const lint*, const lint*, const lint*, const lint*,
                             const double*, const lint*, const lint*, double*, const lint*,
                             lint*, size_t);
extern void scipy_dgemm_64_(const char*, const char*, const lint*, const lint*, const lint*,
                            const double*, const double*, const lint*, const double*,
                            const lint*, const double*, double*, const lint*, size_t, size_t);
extern void scipy_dgemv_64_(const char*, const lint*, const lint*, const double*, const double*,
                            const lint*, const double*, const lint*, const double*, double*,
                            const lint*, size_t);
extern void scipy_dgesv_64_(const lint*, const lint*, double*, const lint*, lint*, double*,
                            const lint*, lint*);
extern void scipy_dgetrf_64_(const lint*, const lint*, double*, const lint*, lint*, lint*);
extern void scipy_dgetri_64_(const lint*, double*, const lint*, const lint*, double*,
                             const lint*, lint*);

void dgbtrf_(lint* m, lint* n, lint* kl, lint* ku, double* ab, lint* ldab, lint* ipiv, lint* info)
{
    scipy_dgbtrf_64_(m, n, kl, ku, ab, ldab, ipiv, info);
}

void dgbtrs_(const char* trans, lint* n, lint* kl, lint* ku, lint* nrhs, double* ab, lint* ldab,
             lint* ipiv, double* b, lint* ldb, lint* info)
{
    scipy_dgbtrs_64_(trans, n, kl, ku, nrhs, ab, ldab, ipiv, b, ldb, info, (size_t)1);
}

int dgemm_(char* transa, char* transb, lint* m, lint* n, lint* k, double* alpha, double* a,
           lint* lda, double* b, lint* ldb, double* beta, double* c, lint* ldc)
{
    scipy_dgemm_64_(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, (size_t)1,
                    (size_t)1);
    return 0;
}

int dgemv_(char* trans, lint* m, lint* n, double* alpha, double* a, lint* lda, double* x,
           lint* incx, double* beta, double* y, lint* incy)
{
    scipy_dgemv_64_(trans, m, n, alpha, a, lda, x, incx, beta, y, incy, (size_t)1);
    return 0;
}

int dgesv_(lint* n, lint* nrhs, double* a, lint* lda, lint* ipiv, double* b, lint* ldb, lint* info)
{
    scipy_dgesv_64_(n, nrhs, a, lda, ipiv, b, ldb, info);
    return 0;
}

int dgetrf_(lint* m, lint* n, double* a, lint* lda, lint* ipiv, lint* info)
{
    scipy_dgetrf_64_(m, n, a, lda, ipiv, info);
    return 0;
}

int dgetri_(lint* n, double* a, lint* lda, lint* ipiv, double* work, lint* lwork, lint* info)
{
    scipy_dgetri_64_(n, a, lda, ipiv, work, lwork, info);
    return 0;
}
