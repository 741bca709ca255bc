/*
 * plasma_ds.h -- mixed-precision solvers (low-precision factor + FP64
 * iterative refinement): SPD (Cholesky) and general (LU), the d/s instance
 * of the reference's zc template include/plasma_zc.h:27-37,58-72.
 */
#ifndef PLASMA_DS_H
#define PLASMA_DS_H

#include "plasma_async.h"
#include "plasma_descriptor.h"
#include "plasma_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * reference compute/zcposv.c:116-271.  Solves A X = B.  A and B are not
 * modified; X receives the solution.  *iter is the number of refinement
 * iterations, or -(itermax+1) = -31 when refinement did not converge and the
 * FP64 factorisation was used instead.  The factor precision follows
 * plasma_set(PlasmaMixedPrecisionMode, ...) (FP32 by default, as in the
 * reference) and the refinement scheme PlasmaRefinement (classical IR by
 * default, as in the reference).
 */
int plasma_dsposv(plasma_enum_t uplo, int n, int nrhs,
                  double *pA, int lda, double *pB, int ldb,
                  double *pX, int ldx, int *iter);

/*
 * reference compute/zcposv.c:363-539.  A, B, X, R are FP64 general
 * descriptors, As and Xs FP32 general descriptors (device memory).  W, Rnorm
 * and Xnorm are host workspaces as in the reference; the GPU build keeps the
 * norms on the device and only copies the per-column values into Rnorm and
 * Xnorm after every convergence test, so W may be NULL.
 */
void plasma_omp_dsposv(plasma_enum_t uplo,
                       plasma_desc_t A, plasma_desc_t B, plasma_desc_t X,
                       plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R,
                       double *W, double *Rnorm, double *Xnorm, int *iter,
                       plasma_sequence_t *sequence, plasma_request_t *request);

/*
 * reference compute/zcgesv.c:106-271.  Solves A X = B for a general square
 * A by an FP32 LU with partial pivoting and FP64 iterative refinement; A and
 * B are not modified, X receives the solution and ipiv (n entries, host
 * memory) the pivots of the factorization used.  *iter as for dsposv
 * (-31: the FP64 LU was used).
 */
int plasma_dsgesv(int n, int nrhs, double *pA, int lda, int *ipiv,
                  double *pB, int ldb, double *pX, int ldx, int *iter);

/*
 * reference compute/zcgesv.c:363-532.  A, B, X, R FP64 and As, Xs FP32
 * general descriptors of one tiling (device memory); ipiv host memory (n
 * entries); work may be NULL (the norms live on the device), Rnorm and
 * Xnorm receive the last columnwise norms when refinement converged.
 */
void plasma_omp_dsgesv(plasma_desc_t A, int *ipiv, plasma_desc_t B, plasma_desc_t X,
                       plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R,
                       double *work, double *Rnorm, double *Xnorm, int *iter,
                       plasma_sequence_t *sequence, plasma_request_t *request);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_DS_H */
