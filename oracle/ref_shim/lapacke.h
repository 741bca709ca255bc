/* Minimal LAPACKE declarations for building the reference PLASMA's SPD path
 * against the OpenBLAS shipped in the image.  Written from the public
 * LAPACKE interface (the column-major constant, the Fortran name mangling
 * macro and the prototypes of the routines the path calls); test
 * infrastructure only. */
#ifndef ORACLE_REF_SHIM_LAPACKE_H
#define ORACLE_REF_SHIM_LAPACKE_H
#include <complex.h>
#ifdef __cplusplus
extern "C" {
#endif

#ifndef lapack_int
#define lapack_int int
#endif
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#ifndef LAPACK_GLOBAL
#define LAPACK_GLOBAL(lcname, UCNAME) lcname##_
#endif
#ifndef lapack_complex_float
#define lapack_complex_float float _Complex
#endif
#ifndef lapack_complex_double
#define lapack_complex_double double _Complex
#endif

lapack_int LAPACKE_dpotrf_work(int layout, char uplo, lapack_int n, double *a,
                               lapack_int lda);
lapack_int LAPACKE_spotrf_work(int layout, char uplo, lapack_int n, float *a,
                               lapack_int lda);
lapack_int LAPACKE_dlacpy_work(int layout, char uplo, lapack_int m, lapack_int n,
                               const double *a, lapack_int lda, double *b,
                               lapack_int ldb);
lapack_int LAPACKE_slacpy_work(int layout, char uplo, lapack_int m, lapack_int n,
                               const float *a, lapack_int lda, float *b,
                               lapack_int ldb);
lapack_int LAPACKE_dlag2s_work(int layout, lapack_int m, lapack_int n,
                               const double *a, lapack_int lda, float *sa,
                               lapack_int ldsa);
lapack_int LAPACKE_slag2d_work(int layout, lapack_int m, lapack_int n,
                               const float *sa, lapack_int ldsa, double *a,
                               lapack_int lda);
lapack_int LAPACKE_dtrtri_work(int layout, char uplo, char diag, lapack_int n,
                               double *a, lapack_int lda);
lapack_int LAPACKE_dlauum_work(int layout, char uplo, lapack_int n, double *a,
                               lapack_int lda);
double LAPACKE_dlamch_work(char cmach);
float LAPACKE_slamch_work(char cmach);
double LAPACKE_dlange_work(int layout, char norm, lapack_int m, lapack_int n,
                           const double *a, lapack_int lda, double *work);
float LAPACKE_slange_work(int layout, char norm, lapack_int m, lapack_int n,
                          const float *a, lapack_int lda, float *work);
double LAPACKE_dlansy_work(int layout, char norm, char uplo, lapack_int n,
                           const double *a, lapack_int lda, double *work);
float LAPACKE_slansy_work(int layout, char norm, char uplo, lapack_int n,
                          const float *a, lapack_int lda, float *work);

#ifdef __cplusplus
}
#endif
#endif
