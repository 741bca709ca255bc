/* Minimal CBLAS declarations for building the reference PLASMA's SPD path
 * against the OpenBLAS shipped in the image.  Written from the public CBLAS
 * interface (enum values and the prototypes of the routines the SPD, LU,
 * band and inverse paths call); test infrastructure only. */
#ifndef ORACLE_REF_SHIM_CBLAS_H
#define ORACLE_REF_SHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
void cblas_sgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, float alpha, const float *a, int lda,
                 const float *b, int ldb, float beta, float *c, int ldc);
void cblas_dsyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                 int n, int k, double alpha, const double *a, int lda,
                 double beta, double *c, int ldc);
void cblas_ssyrk(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                 int n, int k, float alpha, const float *a, int lda,
                 float beta, float *c, int ldc);
void cblas_dtrsm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo,
                 CBLAS_TRANSPOSE ta, CBLAS_DIAG diag, int m, int n,
                 double alpha, const double *a, int lda, double *b, int ldb);
void cblas_strsm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo,
                 CBLAS_TRANSPOSE ta, CBLAS_DIAG diag, int m, int n,
                 float alpha, const float *a, int lda, float *b, int ldb);
void cblas_dsymm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo,
                 int m, int n, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
void cblas_dtrmm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo,
                 CBLAS_TRANSPOSE ta, CBLAS_DIAG diag, int m, int n,
                 double alpha, const double *a, int lda, double *b, int ldb);
void cblas_dswap(int n, double *x, int incx, double *y, int incy);
void cblas_sswap(int n, float *x, int incx, float *y, int incy);
void cblas_dscal(int n, double alpha, double *x, int incx);
void cblas_sscal(int n, float alpha, float *x, int incx);
void cblas_dger(CBLAS_ORDER order, int m, int n, double alpha, const double *x, int incx,
                const double *y, int incy, double *a, int lda);
void cblas_sger(CBLAS_ORDER order, int m, int n, float alpha, const float *x, int incx,
                const float *y, int incy, float *a, int lda);

#ifdef __cplusplus
}
#endif
#endif
