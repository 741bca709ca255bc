/*
 * potri.c -- inverse of an SPD matrix from its Cholesky factor
 * (plasma_dpotri / plasma_omp_dpotri, compute/zpotri.c:65-236) and from the
 * matrix itself (plasma_dpoinv / plasma_omp_dpoinv, compute/zpoinv.c:67-236),
 * with the s variants.
 *
 * Same interface and semantics as the reference: argument codes -1 (uplo),
 * -2 (n), -4 (lda); quick return for n = 0; on exit the uplo triangle of A
 * holds the uplo triangle of inv(A) and the other triangle is left as it
 * was (the reference's tile kernels never touch it); info = i > 0 when the
 * (i,i) element of the factor is zero (potri) or the leading minor of order
 * i is not positive (poinv, from the factorization).
 *
 * The reference inverts the factor (pztrtri, compute/pztrtri.c) and forms
 * the product of the inverse with its transpose (pzlauum,
 * compute/pzlauum.c): 2n^3/3 flops on the triangle.  Here the inverse is
 * the two tile sweeps of potrs applied to the identity,
 * inv(A) = L^-T (L^-1 I): 2n^3 flops, all of them in the sweeps' tile
 * updates, which run as tensor-core GEMMs (the work the reference spreads
 * over trtri, trmm, syrk and lauum tasks becomes two launches per tile
 * step).  The identity and the result live in a scratch slot of the
 * context.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <string.h>

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n);

static int check_async(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
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
    if (A.n == 0)
        return 0;
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    if (A.mb != A.nb || A.m != A.n ||
        A.mb > (A.precision == PlasmaRealDouble ? 512 : 1024)) {
        plasma_error("tile size not supported by the GPU kernels");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return 0;
    }
    return 1;
}

/* inv(A) from the factor held in A (uplo triangle); the call id is that of
 * the request the steps report to */
static void pXpotri(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                    int call, plasma_sequence_t *sequence, plasma_request_t *request)
{
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    const size_t elem = plasma_element_size(A.precision);
    const int mp = A.mt * A.mb;
    void *buf = plasma_scratch(plasma, PLASMA_SLOT_ADJOINT, (size_t)mp * mp * elem);
    if (buf == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_desc_t B;
    plasma_desc_general_init(A.precision, buf, A.mb, A.nb, mp, mp, 0, 0, A.n, A.n, &B);
    cudaMemsetAsync(buf, 0, (size_t)mp * mp * elem, S);
    plasma_cuda_set_diag(S, B, 0, A.n, 1.0);
    plasma_cuda_diag_zero_info(S, st, call, A);
    plasma_pXpotrs(plasma, uplo, A, B, sequence, request);
    plasma_cuda_copy_uplo(S, st, uplo, B, A);
}

static void plasma_omp_Xpotri(plasma_enum_t uplo, plasma_desc_t A,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_async(plasma, uplo, A, sequence, request))
        return;
    if (sequence->status != PlasmaSuccess)
        return;
    int call = plasma_call_begin(plasma, sequence, request);
    pXpotri(plasma, uplo, A, call, sequence, request);
}

static void plasma_omp_Xpoinv(plasma_enum_t uplo, plasma_desc_t A,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_async(plasma, uplo, A, sequence, request))
        return;
    if (sequence->status != PlasmaSuccess)
        return;
    int call = plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrf(plasma, uplo, A, sequence, request, call);
    pXpotri(plasma, uplo, A, call, sequence, request);
}

/* LAPACK-layout drivers (compute/zpotri.c:65-185, zpoinv.c:67-185): the
 * uplo triangle goes up into a kept packed-triangle tile copy and comes
 * back; the other triangle of pA is never touched. */
static int Xdriver(plasma_enum_t prec, plasma_enum_t uplo, int n, void *pA, int lda,
                   int factor)
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
    if (n == 0)
        return PlasmaSuccess;
    if (plasma->device < 0)
        return PlasmaErrorEnvironment;
    if (plasma->tuning)
        plasma_tune_potrf(plasma, prec, n);
    int nb = plasma->nb;

    plasma_desc_t A;
    int retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, prec, uplo, nb, n, n, &A);
    if (retval != PlasmaSuccess)
        return retval;
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
    if (factor)
        plasma_omp_Xpoinv(uplo, A, &sequence, &request);
    else
        plasma_omp_Xpotri(uplo, A, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(A, pA, lda, uplo, &sequence, &request);
    plasma_sequence_wait(&sequence);
    return sequence.status;
}

int plasma_dpotri(plasma_enum_t uplo, int n, double *pA, int lda)
{
    return Xdriver(PlasmaRealDouble, uplo, n, pA, lda, 0);
}

int plasma_spotri(plasma_enum_t uplo, int n, float *pA, int lda)
{
    return Xdriver(PlasmaRealFloat, uplo, n, pA, lda, 0);
}

int plasma_dpoinv(plasma_enum_t uplo, int n, double *pA, int lda)
{
    return Xdriver(PlasmaRealDouble, uplo, n, pA, lda, 1);
}

int plasma_spoinv(plasma_enum_t uplo, int n, float *pA, int lda)
{
    return Xdriver(PlasmaRealFloat, uplo, n, pA, lda, 1);
}

void plasma_omp_dpotri(plasma_enum_t uplo, plasma_desc_t A, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpotri(uplo, A, sequence, request);
}

void plasma_omp_spotri(plasma_enum_t uplo, plasma_desc_t A, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpotri(uplo, A, sequence, request);
}

void plasma_omp_dpoinv(plasma_enum_t uplo, plasma_desc_t A, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpoinv(uplo, A, sequence, request);
}

void plasma_omp_spoinv(plasma_enum_t uplo, plasma_desc_t A, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpoinv(uplo, A, sequence, request);
}
