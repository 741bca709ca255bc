/*
 * adjoint.c -- reverse mode of the tile Cholesky factor and solve.
 *
 * No reference counterpart (PLASMA computes no derivatives).  The entry
 * points follow the library's own conventions: a LAPACK-layout form with
 * host or device pointers and an asynchronous tile form on descriptors.
 *
 * potrf:  A = L L^T, cotangent Lbar of the factor (uplo triangle) ->
 *         Abar = sym(L^-T Phi(L^T Lbar) L^-1), Phi = lower triangle with the
 *         diagonal halved.  Tile steps: P = L^T Lbar on the lower triangle
 *         (masked tensor-core GEMM, K clipped to the non-zero band),
 *         W = Phi(P)^T, W <- L^-T W (tile sweep, n right-hand sides),
 *         W <- W^T, W <- L^-T W, Abar = (W + W^T)/2.  Work: n^3/3 for P,
 *         n^3 for the two triangular solves with full right-hand sides.
 * potrs:  X = A^-1 B, cotangent Xbar -> Bbar = A^-1 Xbar (the library's
 *         potrs) and Lbar -= tril((Bbar X^T + X Bbar^T) L), formed as
 *         Bbar (X^T L) + X (Bbar^T L): 4 n^2 nrhs flops.
 * Upper storage (A = U^T U) works on the logical lower view L = U^T; the
 * cotangents are then Ubar = Lbar^T.
 */
#include "../internal.h"

#include <string.h>

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);

static plasma_view_t view(plasma_desc_t D, int trans, int tri)
{
    plasma_view_t v;
    memset(&v, 0, sizeof(v));
    v.D = D;
    v.trans = trans;
    v.tri = tri;
    return v;
}

/* The logical lower factor L held in D with storage uplo, or its transpose. */
static plasma_view_t factor_view(plasma_desc_t D, plasma_enum_t uplo, int transpose)
{
    if (uplo == PlasmaLower)
        return view(D, transpose, 1);
    return view(D, !transpose, 2);        /* L = U^T */
}

static int check_tile(plasma_context_t *plasma, plasma_enum_t uplo,
                      plasma_desc_t A, plasma_sequence_t *sequence,
                      plasma_request_t *request)
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
    if (plasma_desc_check(A) != PlasmaSuccess || A.m != A.n) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    if (A.mb != A.nb) {
        plasma_error("square tiles required");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return 0;
    }
    return sequence->status == PlasmaSuccess;
}

/* Abar from (L, Lbar): L and Lbar n x n with the factor and its cotangent in
 * the uplo triangle; on return Lbar holds the full symmetric Abar. */
void plasma_pXpotrf_adjoint(plasma_context_t *plasma, plasma_enum_t uplo,
                            plasma_desc_t L, plasma_desc_t Lbar,
                            plasma_sequence_t *sequence, plasma_request_t *request)
{
    const int n = L.m;
    if (n == 0)
        return;
    cudaStream_t s = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    const size_t elem = plasma_element_size(L.precision);
    const int mb = L.mb;
    const int ldw = ((n + mb - 1) / mb) * mb;
    const size_t wbytes = (size_t)ldw * ldw * elem;
    char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_ADJOINT, 2 * wbytes);
    void *winv = plasma_scratch(plasma, PLASMA_SLOT_WORK,
                                (size_t)L.mt * mb * mb * elem);
    if (buf == NULL || winv == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_desc_t W1, W2;
    plasma_desc_general_init(L.precision, buf, mb, mb, ldw, ldw, 0, 0, n, n, &W1);
    plasma_desc_general_init(L.precision, buf + wbytes, mb, mb, ldw, ldw, 0, 0, n, n, &W2);

    /* P = L^T Lbar on the lower triangle, zero above */
    plasma_view_t lbar = uplo == PlasmaLower ? view(Lbar, 0, 1) : view(Lbar, 1, 2);
    plasma_cuda_gemm_view(s, st, n, n, n, 1.0, factor_view(L, uplo, 1), lbar, 0.0,
                          view(W1, 0, 0), 1, 1);
    /* W2 = Phi(P)^T */
    plasma_view_t phi = view(W1, 1, 1);
    phi.diag_scale = 1;
    plasma_cuda_copy_view(s, st, n, n, phi, view(W2, 0, 0));
    /* W2 = L^-T Phi(P)^T = (Phi(P) L^-1)^T */
    plasma_cuda_trsm_sweep(s, st, uplo, PlasmaTrans, L, W2, winv, 0);
    /* W1 = Phi(P) L^-1, then W1 = L^-T Phi(P) L^-1 */
    plasma_cuda_copy_view(s, st, n, n, view(W2, 1, 0), view(W1, 0, 0));
    plasma_cuda_trsm_sweep(s, st, uplo, PlasmaTrans, L, W1, winv, 1);
    /* Abar = sym(W1) */
    plasma_cuda_symmetrize(s, st, n, view(W1, 0, 0), view(Lbar, 0, 0));
}

/* Bbar = A^-1 Xbar in place of Xbar; Lbar (uplo triangle) -= the factor
 * cotangent of the solve. */
void plasma_pXpotrs_adjoint(plasma_context_t *plasma, plasma_enum_t uplo,
                            plasma_desc_t L, plasma_desc_t X, plasma_desc_t Xbar,
                            plasma_desc_t Lbar, plasma_sequence_t *sequence,
                            plasma_request_t *request)
{
    const int n = L.m, nrhs = X.n;
    if (n == 0 || nrhs == 0)
        return;
    cudaStream_t s = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    plasma_pXpotrs(plasma, uplo, L, Xbar, sequence, request);

    const size_t elem = plasma_element_size(L.precision);
    const int mb = L.mb;
    const int ldu = ((nrhs + mb - 1) / mb) * mb, ncol = ((n + mb - 1) / mb) * mb;
    const size_t ubytes = (size_t)ldu * ncol * elem;
    char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_ADJOINT, 2 * ubytes);
    if (buf == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_desc_t U1, U2;
    plasma_desc_general_init(L.precision, buf, mb, mb, ldu, ncol, 0, 0, nrhs, n, &U1);
    plasma_desc_general_init(L.precision, buf + ubytes, mb, mb, ldu, ncol, 0, 0, nrhs, n, &U2);
    plasma_view_t lv = factor_view(L, uplo, 0);
    /* U1 = X^T L, U2 = Bbar^T L  (nrhs x n) */
    plasma_cuda_gemm_view(s, st, nrhs, n, n, 1.0, view(X, 1, 0), lv, 0.0,
                          view(U1, 0, 0), 0, 0);
    plasma_cuda_gemm_view(s, st, nrhs, n, n, 1.0, view(Xbar, 1, 0), lv, 0.0,
                          view(U2, 0, 0), 0, 0);
    if (uplo == PlasmaLower) {
        /* Lbar -= Bbar U1 + X U2 on the lower triangle */
        plasma_cuda_gemm_view(s, st, n, n, nrhs, -1.0, view(Xbar, 0, 0), view(U1, 0, 0),
                              1.0, view(Lbar, 0, 0), 1, 0);
        plasma_cuda_gemm_view(s, st, n, n, nrhs, -1.0, view(X, 0, 0), view(U2, 0, 0),
                              1.0, view(Lbar, 0, 0), 1, 0);
    } else {
        /* Ubar = Lbar^T -= U1^T Bbar^T + U2^T X^T on the upper triangle */
        plasma_cuda_gemm_view(s, st, n, n, nrhs, -1.0, view(U1, 1, 0), view(Xbar, 1, 0),
                              1.0, view(Lbar, 0, 0), 2, 0);
        plasma_cuda_gemm_view(s, st, n, n, nrhs, -1.0, view(U2, 1, 0), view(X, 1, 0),
                              1.0, view(Lbar, 0, 0), 2, 0);
    }
}

/* ---------------------------------------------------------------- tile API */

static void omp_potrf_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t Lbar,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_tile(plasma, uplo, L, sequence, request))
        return;
    if (plasma_desc_check(Lbar) != PlasmaSuccess || Lbar.m != L.m || Lbar.n != L.n ||
        Lbar.type != PlasmaGeneral || Lbar.precision != L.precision) {
        plasma_error("invalid Lbar");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrf_adjoint(plasma, uplo, L, Lbar, sequence, request);
}

static void omp_potrs_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t X,
                              plasma_desc_t Xbar, plasma_desc_t Lbar,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_tile(plasma, uplo, L, sequence, request))
        return;
    if (plasma_desc_check(X) != PlasmaSuccess || plasma_desc_check(Xbar) != PlasmaSuccess ||
        X.m != L.m || Xbar.m != L.m || Xbar.n != X.n || X.mb != L.mb || Xbar.mb != L.mb ||
        X.precision != L.precision || Xbar.precision != L.precision) {
        plasma_error("invalid X or Xbar");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (plasma_desc_check(Lbar) != PlasmaSuccess || Lbar.m != L.m || Lbar.n != L.n ||
        Lbar.precision != L.precision) {
        plasma_error("invalid Lbar");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrs_adjoint(plasma, uplo, L, X, Xbar, Lbar, sequence, request);
}

void plasma_omp_dpotrf_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    omp_potrf_adjoint(uplo, L, Lbar, sequence, request);
}

void plasma_omp_spotrf_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    omp_potrf_adjoint(uplo, L, Lbar, sequence, request);
}

void plasma_omp_dpotrs_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t X,
                               plasma_desc_t Xbar, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    omp_potrs_adjoint(uplo, L, X, Xbar, Lbar, sequence, request);
}

void plasma_omp_spotrs_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t X,
                               plasma_desc_t Xbar, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    omp_potrs_adjoint(uplo, L, X, Xbar, Lbar, sequence, request);
}

/* ------------------------------------------------------ LAPACK-layout API */

static int Xpotrf_adjoint(plasma_enum_t prec, plasma_enum_t uplo, int n,
                          const void *pL, int ldl, void *pLbar, int ldlbar)
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
    if (ldl < imax(1, n)) {
        plasma_error("illegal value of ldl");
        return -4;
    }
    if (ldlbar < imax(1, n)) {
        plasma_error("illegal value of ldlbar");
        return -6;
    }
    if (n == 0)
        return PlasmaSuccess;
    const int nb = plasma->nb;
    plasma_desc_t L, Lbar;
    int rc = plasma_desc_general_create(prec, nb, nb, n, n, 0, 0, n, n, &L);
    if (rc != PlasmaSuccess)
        return rc;
    rc = plasma_desc_general_create(prec, nb, nb, n, n, 0, 0, n, n, &Lbar);
    if (rc != PlasmaSuccess) {
        plasma_desc_destroy(&L);
        return rc;
    }
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);
    plasma_omp_Xlapack2desc(pL, ldl, L, uplo, &sequence, &request);
    plasma_omp_Xlapack2desc(pLbar, ldlbar, Lbar, uplo, &sequence, &request);
    omp_potrf_adjoint(uplo, L, Lbar, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(Lbar, pLbar, ldlbar, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_desc_destroy(&L);
    plasma_desc_destroy(&Lbar);
    return sequence.status;
}

static int Xpotrs_adjoint(plasma_enum_t prec, plasma_enum_t uplo, int n, int nrhs,
                          const void *pL, int ldl, const void *pX, int ldx,
                          void *pXbar, int ldxbar, void *pLbar, int ldlbar)
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
    if (nrhs < 0) {
        plasma_error("illegal value of nrhs");
        return -3;
    }
    if (ldl < imax(1, n)) {
        plasma_error("illegal value of ldl");
        return -5;
    }
    if (ldx < imax(1, n)) {
        plasma_error("illegal value of ldx");
        return -7;
    }
    if (ldxbar < imax(1, n)) {
        plasma_error("illegal value of ldxbar");
        return -9;
    }
    if (ldlbar < imax(1, n)) {
        plasma_error("illegal value of ldlbar");
        return -11;
    }
    if (imin(n, nrhs) == 0)
        return PlasmaSuccess;
    const int nb = plasma->nb;
    plasma_desc_t L, X, Xbar, Lbar;
    int rc = plasma_desc_general_create(prec, nb, nb, n, n, 0, 0, n, n, &L);
    if (rc == PlasmaSuccess)
        rc = plasma_desc_general_create(prec, nb, nb, n, nrhs, 0, 0, n, nrhs, &X);
    if (rc == PlasmaSuccess)
        rc = plasma_desc_general_create(prec, nb, nb, n, nrhs, 0, 0, n, nrhs, &Xbar);
    if (rc == PlasmaSuccess)
        rc = plasma_desc_general_create(prec, nb, nb, n, n, 0, 0, n, n, &Lbar);
    if (rc != PlasmaSuccess) {
        plasma_desc_destroy(&L);
        plasma_desc_destroy(&X);
        plasma_desc_destroy(&Xbar);
        plasma_desc_destroy(&Lbar);
        return rc;
    }
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);
    plasma_omp_Xlapack2desc(pL, ldl, L, uplo, &sequence, &request);
    plasma_omp_Xlapack2desc(pX, ldx, X, PlasmaGeneral, &sequence, &request);
    plasma_omp_Xlapack2desc(pXbar, ldxbar, Xbar, PlasmaGeneral, &sequence, &request);
    plasma_omp_Xlapack2desc(pLbar, ldlbar, Lbar, uplo, &sequence, &request);
    omp_potrs_adjoint(uplo, L, X, Xbar, Lbar, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(Xbar, pXbar, ldxbar, PlasmaGeneral, &sequence, &request);
    plasma_omp_Xdesc2lapack(Lbar, pLbar, ldlbar, uplo, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_desc_destroy(&L);
    plasma_desc_destroy(&X);
    plasma_desc_destroy(&Xbar);
    plasma_desc_destroy(&Lbar);
    return sequence.status;
}

int plasma_dpotrf_adjoint(plasma_enum_t uplo, int n, const double *pL, int ldl,
                          double *pLbar, int ldlbar)
{
    return Xpotrf_adjoint(PlasmaRealDouble, uplo, n, pL, ldl, pLbar, ldlbar);
}

int plasma_spotrf_adjoint(plasma_enum_t uplo, int n, const float *pL, int ldl,
                          float *pLbar, int ldlbar)
{
    return Xpotrf_adjoint(PlasmaRealFloat, uplo, n, pL, ldl, pLbar, ldlbar);
}

int plasma_dpotrs_adjoint(plasma_enum_t uplo, int n, int nrhs, const double *pL, int ldl,
                          const double *pX, int ldx, double *pXbar, int ldxbar,
                          double *pLbar, int ldlbar)
{
    return Xpotrs_adjoint(PlasmaRealDouble, uplo, n, nrhs, pL, ldl, pX, ldx, pXbar,
                          ldxbar, pLbar, ldlbar);
}

int plasma_spotrs_adjoint(plasma_enum_t uplo, int n, int nrhs, const float *pL, int ldl,
                          const float *pX, int ldx, float *pXbar, int ldxbar,
                          float *pLbar, int ldlbar)
{
    return Xpotrs_adjoint(PlasmaRealFloat, uplo, n, nrhs, pL, ldl, pX, ldx, pXbar,
                          ldxbar, pLbar, ldlbar);
}
