/*
 * potrf.c -- Cholesky factorisation drivers, double and single precision.
 *
 * plasma_{d,s}potrf follow the reference's compute/zpotrf.c:74-150: argument
 * checks (-1 uplo, -2 n, -4 lda), quick return, tuning of nb
 * (plasma_tune_potrf), a packed-triangular descriptor, tr2desc -> async
 * factorisation -> desc2tr, and the sequence status as return value.
 * plasma_omp_{d,s}potrf follow :206-246.  The work is enqueued on the
 * context stream; the LAPACK-layout routine waits for it.
 */
#include "../internal.h"

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n);

void plasma_omp_Xpotrf(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        /* the reference exits here; a library call returns instead */
        plasma_error("PLASMA not initialized");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return;
    }
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (plasma_desc_check(A) != PlasmaSuccess) {
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        plasma_error("invalid A");
        return;
    }
    if (A.m == 0)
        return;
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return;
    }
    if (A.mb != A.nb || A.mb > (A.precision == PlasmaRealDouble ? 512 : 1024)) {
        plasma_error("tile size not supported by the GPU kernels");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return;
    }
    int call = plasma_call_begin(plasma, sequence, request);
    /* GPU-build extension: an FP32 factorisation follows
     * PlasmaMixedPrecisionMode (TF32 / BF16 products on the tensor cores,
     * FP32 accumulation); the default FP32 mode is plain FP32 arithmetic. */
    int mode = A.precision == PlasmaRealFloat ? plasma->mixed_mode : 0;
    if (mode == PlasmaFactorAuto)
        mode = PlasmaFactorTF32;
    plasma_pXpotrf_mode(plasma, uplo, A, sequence, request, call, mode);
}

static int Xpotrf(plasma_enum_t prec, plasma_enum_t uplo, int n, void *pA,
                  int lda)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        return -1;
    }
    if (n < 0) {
        plasma_error("illegal value of n");
        return -2;
    }
    if (lda < imax(1, n)) {
        plasma_error("illegal value of lda");
        return -4;
    }
    if (imax(n, 0) == 0)
        return PlasmaSuccess;

    if (plasma->tuning)
        plasma_tune_potrf(plasma, prec, n);
    int nb = plasma->nb;

    /* An upper-stored matrix is factored through lower tiles: its tile
     * copy holds U^T (the transpose of the stored triangle), the lower
     * factor L of that copy is the transpose of the upper factor U, and it
     * goes back transposed.  The trailing updates then run on the tensor
     * cores, which take lower tiles. */
    const int via_lower = uplo == PlasmaUpper;
    plasma_desc_t A;
    /* the tile copy lives in a slot the context keeps between calls */
    int retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, prec,
                                  via_lower ? PlasmaLower : uplo, nb, n, n, &A);
    if (retval != PlasmaSuccess) {
        plasma_error("tile copy of A failed");
        return retval;
    }
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    if (via_lower)
        plasma_omp_Xlapack2desc_t(pA, lda, A, &sequence, &request);
    else
        plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
    plasma_omp_Xpotrf(via_lower ? PlasmaLower : uplo, A, &sequence, &request);
    /* After a failure the reference's desc2tr tasks see the failed sequence
     * and skip, leaving pA as it was; waiting here makes that exact. */
    plasma_sequence_wait(&sequence);
    if (via_lower)
        plasma_omp_Xdesc2lapack_t(A, pA, lda, &sequence, &request);
    else
        plasma_omp_Xdesc2lapack(A, pA, lda, uplo, &sequence, &request);
    plasma_sequence_wait(&sequence);
    return sequence.status;
}

int plasma_dpotrf(plasma_enum_t uplo, int n, double *pA, int lda)
{
    return Xpotrf(PlasmaRealDouble, uplo, n, pA, lda);
}

int plasma_spotrf(plasma_enum_t uplo, int n, float *pA, int lda)
{
    return Xpotrf(PlasmaRealFloat, uplo, n, pA, lda);
}

void plasma_omp_dpotrf(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpotrf(uplo, A, sequence, request);
}

void plasma_omp_spotrf(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpotrf(uplo, A, sequence, request);
}
