/*
 * plasma_d.h -- double-precision SPD routines of the PLASMA C API.
 *
 * Each prototype replaces the reference routine cited beside it (the z
 * template that the reference's code generator turns into the d routine).
 * Semantics kept: argument checks return -i for the i-th illegal argument,
 * PlasmaErrorNotInitialized without plasma_init(), and +i for the order of the
 * first non positive definite leading minor.
 *
 * GPU build: pA/pB may be host or device pointers (detected per call); tile
 * descriptors passed to plasma_omp_* hold device memory.
 */
#ifndef PLASMA_D_H
#define PLASMA_D_H

#include "plasma_async.h"
#include "plasma_descriptor.h"
#include "plasma_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference compute/zpotrf.c:74-150 */
int plasma_dpotrf(plasma_enum_t uplo, int n, double *pA, int lda);
/* reference compute/zpotrs.c:77-172 */
int plasma_dpotrs(plasma_enum_t uplo, int n, int nrhs,
                  double *pA, int lda, double *pB, int ldb);
/* reference compute/zposv.c:90-186 */
int plasma_dposv(plasma_enum_t uplo, int n, int nrhs,
                 double *pA, int lda, double *pB, int ldb);

/* reference compute/zpotri.c:65-185: inverse from the Cholesky factor */
int plasma_dpotri(plasma_enum_t uplo, int n, double *pA, int lda);
/* reference compute/zpoinv.c:67-185: inverse of an SPD matrix */
int plasma_dpoinv(plasma_enum_t uplo, int n, double *pA, int lda);

/* reference compute/zpotri.c:187-236 */
void plasma_omp_dpotri(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zpoinv.c:187-236 */
void plasma_omp_dpoinv(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request);

/* reference compute/zpbtrf.c:77-158: Cholesky of an SPD band matrix in
 * LAPACK band storage (AB(kd+1+i-j,j) upper, AB(1+i-j,j) lower) */
int plasma_dpbtrf(plasma_enum_t uplo, int n, int kd, double *pAB, int ldab);
/* reference compute/zpbtrs.c:81-182: solve with the band factor */
int plasma_dpbtrs(plasma_enum_t uplo, int n, int kd, int nrhs,
                  double *pAB, int ldab, double *pB, int ldb);
/* reference compute/zpbsv.c:92-193: factor and solve */
int plasma_dpbsv(plasma_enum_t uplo, int n, int kd, int nrhs,
                 double *pAB, int ldab, double *pB, int ldb);

/* reference compute/zpbtrf.c:202-242 (AB: a band descriptor) */
void plasma_omp_dpbtrf(plasma_enum_t uplo, plasma_desc_t AB,
                       plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zpbtrs.c:236-295 */
void plasma_omp_dpbtrs(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zpbsv.c:242-302 */
void plasma_omp_dpbsv(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zpb2desc.c (pAB host or device) */
void plasma_omp_dpb2desc(double *pAB, int ldab, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zdesc2pb.c */
void plasma_omp_ddesc2pb(plasma_desc_t A, double *pAB, int ldab,
                         plasma_sequence_t *sequence, plasma_request_t *request);

/* reference compute/zpotrf.c:206-246 */
void plasma_omp_dpotrf(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zpotrs.c:226-283 */
void plasma_omp_dpotrs(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zposv.c:244-301 */
void plasma_omp_dposv(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request);

/* reference compute/zge2desc.c:27-68 (pA host or device) */
void plasma_omp_dge2desc(double *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zdesc2ge.c */
void plasma_omp_ddesc2ge(plasma_desc_t A, double *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/ztr2desc.c */
void plasma_omp_dtr2desc(double *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request);
/* reference compute/zdesc2tr.c */
void plasma_omp_ddesc2tr(plasma_desc_t A, double *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_D_H */
