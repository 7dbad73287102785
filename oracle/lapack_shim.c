/*
 * Test infrastructure only: LAPACK entry points for the reference build.
 *
 * The reference solves every kriging system with LAPACK dpotrf/dpotrs
 * (src/geo_bsd/hpgl/my_kriging_weights.h:147,162,284,302-303). This image has
 * no system LAPACK, so these two symbols forward to the LP64 routines that
 * SciPy's bundled OpenBLAS exports under the `scipy_` prefix. Only exported
 * names of an installed library are used.
 */
void scipy_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info);
void scipy_dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a,
                   const int *lda, double *b, const int *ldb, int *info);

void dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info)
{
    scipy_dpotrf_(uplo, n, a, lda, info);
}

void dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a,
             const int *lda, double *b, const int *ldb, int *info)
{
    scipy_dpotrs_(uplo, n, nrhs, a, lda, b, ldb, info);
}
