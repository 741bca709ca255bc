/*
 * plasma_core_blas.h -- the reference's CPU tile kernels of the
 * kernel-substitution interface, d and s instances of
 * include/plasma_core_blas_z.h:57-61 (geadd), :70-75 (gemm), :153-157
 * (lacpy), :173-177 (lange), :185-189 (lansy), :266-269 (potrf), :271-276
 * (symm), :285-289 (syrk), :304-309 (trsm), :407-410 (omp_dzamax) and
 * include/plasma_core_blas_zc.h:24-32 (lag2c / clag2z).  Host-memory
 * kernels with BLAS / LAPACK semantics, exported by libplasma_core_blas.so
 * (a compatibility library; libplasma_b200.so does not use it).
 */
#ifndef PLASMA_CORE_BLAS_H
#define PLASMA_CORE_BLAS_H

#include "plasma_async.h"
#include "plasma_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PLASMA_CORE_BLAS_DECLS(P, T)                                                       \
    int plasma_core_##P##potrf(plasma_enum_t uplo, int n, T *A, int lda);                  \
    void plasma_core_##P##trsm(plasma_enum_t side, plasma_enum_t uplo, plasma_enum_t transa, \
                               plasma_enum_t diag, int m, int n, T alpha, const T *A,      \
                               int lda, T *B, int ldb);                                    \
    void plasma_core_##P##syrk(plasma_enum_t uplo, plasma_enum_t trans, int n, int k,      \
                               T alpha, const T *A, int lda, T beta, T *C, int ldc);       \
    void plasma_core_##P##gemm(plasma_enum_t transa, plasma_enum_t transb, int m, int n,   \
                               int k, T alpha, const T *A, int lda, const T *B, int ldb,   \
                               T beta, T *C, int ldc);                                     \
    void plasma_core_##P##symm(plasma_enum_t side, plasma_enum_t uplo, int m, int n,       \
                               T alpha, const T *A, int lda, const T *B, int ldb, T beta,  \
                               T *C, int ldc);                                             \
    void plasma_core_##P##lacpy(plasma_enum_t uplo, plasma_enum_t transa, int m, int n,    \
                                const T *A, int lda, T *B, int ldb);                       \
    int plasma_core_##P##geadd(plasma_enum_t transa, int m, int n, T alpha, const T *A,    \
                               int lda, T beta, T *B, int ldb);                            \
    void plasma_core_##P##lange(plasma_enum_t norm, int m, int n, const T *A, int lda,     \
                                double *work, double *value);                              \
    void plasma_core_##P##lansy(plasma_enum_t norm, plasma_enum_t uplo, int n, const T *A, \
                                int lda, double *work, double *value);                     \
    void plasma_core_omp_##P##amax(int colrow, int m, int n, const T *A, int lda,          \
                                   double *values, plasma_sequence_t *sequence,            \
                                   plasma_request_t *request);

PLASMA_CORE_BLAS_DECLS(d, double)
PLASMA_CORE_BLAS_DECLS(s, float)

int plasma_core_dlag2s(int m, int n, const double *A, int lda, float *As, int ldas);
void plasma_core_slag2d(int m, int n, const float *As, int ldas, double *A, int lda);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_CORE_BLAS_H */
