/*
 * posv.c -- plasma_{d,s}potrs and plasma_{d,s}posv with their async forms.
 *
 * potrs follows the reference's compute/zpotrs.c:77-172 (A in a general
 * descriptor, -1/-2/-3/-5/-7 argument codes, quick return when
 * max(n, nrhs) == 0, only B written back) and :226-283 (two pdtrsm sweeps,
 * Left/Lower NoTrans then Trans, or Upper Trans then NoTrans).
 * posv follows compute/zposv.c:90-186 (A packed triangular, quick return when
 * min(n, nrhs) == 0, A and B written back) and :244-301 (pdpotrf + 2 pdtrsm).
 */
#include "../internal.h"

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xpotrf(plasma_enum_t uplo, plasma_desc_t A,
                       plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n);
void plasma_tune_trsm(plasma_context_t *plasma, plasma_enum_t dtyp, int m,
                      int n);

/* Both triangular sweeps with the factor held in A (any storage uplo). */
void plasma_pXpotrs(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_desc_t B,
                    plasma_sequence_t *sequence, plasma_request_t *request)
{
    if (sequence->status != PlasmaSuccess)
        return;
    size_t elem = plasma_element_size(A.precision);
    size_t wb = (size_t)A.mt * A.mb * A.mb * elem;
    size_t wv = plasma_cuda_trsv_w_bytes(A);
    void *W = plasma_scratch(plasma, PLASMA_SLOT_WORK, wb > wv ? wb : wv);
    if (W == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    /* one right-hand side: B is a contiguous vector, solved by the
     * one-launch sweeps; up to 32: the multi-column one-launch sweeps, 16
     * columns at a time; otherwise step-by-step tile sweeps */
    if (B.n == 1 && B.nt == 1 && B.i == 0 && B.j == 0 && B.gn == 1 &&
        plasma_sweep_reserve(plasma, A)) {
        plasma_cuda_trtri_blocks(plasma->stream, plasma->dstat, uplo, A, W);
        plasma_sweep(plasma, uplo, 0, A, W, B.matrix);
        plasma_sweep(plasma, uplo, 1, A, W, B.matrix);
        return;
    }
    if (B.n >= 2 && B.n <= 32 && B.i == 0 && B.j == 0 && B.m == A.m &&
        B.precision == A.precision && plasma_cuda_trsv_block(A) > 0 &&
        plasma_sweep_reserve(plasma, A)) {
        plasma_cuda_trtri_blocks(plasma->stream, plasma->dstat, uplo, A, W);
        for (int c0 = 0; c0 < B.n; c0 += 16) {
            const int nc = imin(16, B.n - c0);
            plasma_sweep_rows(plasma, uplo, 0, A, W, B, c0, nc);
            plasma_sweep_rows(plasma, uplo, 1, A, W, B, c0, nc);
        }
        return;
    }
    plasma_cuda_trsm_sweep(plasma->stream, plasma->dstat, uplo, PlasmaNoTrans,
                           A, B, W, 0);
    plasma_cuda_trsm_sweep(plasma->stream, plasma->dstat, uplo, PlasmaTrans,
                           A, B, W, 1);
}

static int check_async(plasma_context_t *plasma, plasma_enum_t uplo,
                       plasma_desc_t A, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return 0;
    }
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma_desc_check(A) != PlasmaSuccess) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma_desc_check(B) != PlasmaSuccess) {
        plasma_error("invalid B");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (A.n == 0 || B.n == 0)
        return 0;
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    if (A.mb != A.nb || B.mb != A.mb ||
        A.mb > (A.precision == PlasmaRealDouble ? 512 : 1024)) {
        plasma_error("tile size not supported by the GPU kernels");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return 0;
    }
    return 1;
}

void plasma_omp_Xpotrs(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_async(plasma, uplo, A, B, sequence, request))
        return;
    plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrs(plasma, uplo, A, B, sequence, request);
}

void plasma_omp_Xposv(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_async(plasma, uplo, A, B, sequence, request))
        return;
    int call = plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrf(plasma, uplo, A, sequence, request, call);
    plasma_pXpotrs(plasma, uplo, A, B, sequence, request);
}

static int check_lapack(plasma_enum_t uplo, int n, int nrhs, int lda, int ldb)
{
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        return -1;
    }
    if (n < 0) {
        plasma_error("illegal value of n");
        return -2;
    }
    if (nrhs < 0) {
        plasma_error("illegal value of nrhs");
        return -3;
    }
    if (lda < imax(1, n)) {
        plasma_error("illegal value of lda");
        return -5;
    }
    if (ldb < imax(1, n)) {
        plasma_error("illegal value of ldb");
        return -7;
    }
    return 0;
}

static int Xpotrs(plasma_enum_t prec, plasma_enum_t uplo, int n, int nrhs,
                  void *pA, int lda, void *pB, int ldb)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    int info = check_lapack(uplo, n, nrhs, lda, ldb);
    if (info != 0)
        return info;
    if (imax(n, nrhs) == 0)
        return PlasmaSuccess;
    if (plasma->tuning)
        plasma_tune_trsm(plasma, prec, n, n);
    int nb = plasma->nb;

    plasma_desc_t A, B;
    /* the tile copy of A lives in a slot the context keeps between calls */
    int retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, prec, PlasmaGeneral, nb, n, n,
                                  &A);
    if (retval != PlasmaSuccess)
        return retval;
    retval = plasma_desc_general_create(prec, nb, nb, n, nrhs, 0, 0, n, nrhs, &B);
    if (retval != PlasmaSuccess)
        return retval;
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    /* only the uplo triangle of the factor is referenced */
    plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
    plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    plasma_omp_Xpotrs(uplo, A, B, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(B, pB, ldb, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);

    plasma_desc_destroy(&B);
    return sequence.status;
}

static int Xposv(plasma_enum_t prec, plasma_enum_t uplo, int n, int nrhs,
                 void *pA, int lda, void *pB, int ldb)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    int info = check_lapack(uplo, n, nrhs, lda, ldb);
    if (info != 0)
        return info;
    if (imin(n, nrhs) == 0)
        return PlasmaSuccess;
    if (plasma->tuning)
        plasma_tune_potrf(plasma, prec, n);
    int nb = plasma->nb;

    /* an upper-stored matrix goes through lower tiles, as in Xpotrf; its
     * host staging buffer keeps the untouched strictly lower part of the
     * diagonal blocks for the way back, so B is converted before it and
     * after it */
    const int via_lower = uplo == PlasmaUpper;
    plasma_desc_t A, B;
    /* the tile copy of A lives in a slot the context keeps between calls */
    int retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, prec,
                                  via_lower ? PlasmaLower : uplo, nb, n, n, &A);
    if (retval != PlasmaSuccess)
        return retval;
    retval = plasma_desc_general_create(prec, nb, nb, n, nrhs, 0, 0, n, nrhs, &B);
    if (retval != PlasmaSuccess)
        return retval;
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    if (via_lower) {
        plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
        plasma_omp_Xlapack2desc_t(pA, lda, A, &sequence, &request);
    } else {
        plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
        plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    }
    plasma_omp_Xposv(via_lower ? PlasmaLower : uplo, A, B, &sequence, &request);
    plasma_sequence_wait(&sequence);
    if (via_lower)
        plasma_omp_Xdesc2lapack_t(A, pA, lda, &sequence, &request);
    else
        plasma_omp_Xdesc2lapack(A, pA, lda, uplo, &sequence, &request);
    plasma_omp_Xdesc2lapack(B, pB, ldb, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);

    plasma_desc_destroy(&B);
    return sequence.status;
}

int plasma_dpotrs(plasma_enum_t uplo, int n, int nrhs, double *pA, int lda,
                  double *pB, int ldb)
{
    return Xpotrs(PlasmaRealDouble, uplo, n, nrhs, pA, lda, pB, ldb);
}

int plasma_spotrs(plasma_enum_t uplo, int n, int nrhs, float *pA, int lda,
                  float *pB, int ldb)
{
    return Xpotrs(PlasmaRealFloat, uplo, n, nrhs, pA, lda, pB, ldb);
}

int plasma_dposv(plasma_enum_t uplo, int n, int nrhs, double *pA, int lda,
                 double *pB, int ldb)
{
    return Xposv(PlasmaRealDouble, uplo, n, nrhs, pA, lda, pB, ldb);
}

int plasma_sposv(plasma_enum_t uplo, int n, int nrhs, float *pA, int lda,
                 float *pB, int ldb)
{
    return Xposv(PlasmaRealFloat, uplo, n, nrhs, pA, lda, pB, ldb);
}

void plasma_omp_dpotrs(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpotrs(uplo, A, B, sequence, request);
}

void plasma_omp_spotrs(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpotrs(uplo, A, B, sequence, request);
}

void plasma_omp_dposv(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xposv(uplo, A, B, sequence, request);
}

void plasma_omp_sposv(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xposv(uplo, A, B, sequence, request);
}
