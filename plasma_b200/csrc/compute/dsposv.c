/*
 * dsposv.c -- mixed-precision SPD solver: low-precision Cholesky factor,
 * FP64 iterative refinement, FP64 fallback.
 *
 * Follows the reference's compute/zcposv.c:
 *   plasma_dsposv      :116-271 (argument codes -1,-2,-3,-5,-7,-9; iter = 0
 *                       and quick return when min(n, nrhs) == 0)
 *   conv()             :275-287 (every column: Rnorm <= Xnorm * cte)
 *   plasma_omp_dsposv  :363-539: Anorm = lansy_inf(A); Xs = lag2s(B);
 *                       As = lag2s(A); spotrf(As); two strsm; X = slag2d(Xs);
 *                       R = B - A X; test with cte = Anorm*eps*sqrt(n);
 *                       up to itermax = 30 refinement steps; otherwise
 *                       iter = -31 and the FP64 potrf + two trsm.
 *
 * Deliberate differences (also listed in the design notes):
 *  - When the low-precision factorisation or a conversion fails, the reference
 *    marks the whole sequence as failed and returns that info with iter = -31
 *    without solving (an SPD matrix that is not SPD in FP32 is reported as
 *    not positive definite).  Here the solver falls back to the FP64
 *    factorisation, as LAPACK's dsposv -- the reference tester's oracle -- does,
 *    and returns the FP64 info (iter = -31).
 *  - Only the uplo triangle of A is converted (the reference converts the full
 *    general matrix, with a "TODO: need zlat2c" note at zcposv.c:447).
 *  - Extended factor precisions and GMRES-IR are available through
 *    PlasmaMixedPrecisionMode / PlasmaRefinement (defaults match the
 *    reference: FP32 factor, classical IR).
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n);

#define ITERMAX 30

static int conv(const double *Rnorm, const double *Xnorm, int n, double cte)
{
    for (int i = 0; i < n; i++)
        if (!(Rnorm[i] <= Xnorm[i] * cte))
            return 0;
    return 1;
}

/* Reads the device status (after a stream sync); returns it and clears it so
 * that the next phase starts clean. */
static int take_status(plasma_context_t *plasma)
{
    cudaStreamSynchronize(plasma->stream);
    cudaMemcpy(plasma->hstat, plasma->dstat, sizeof(plasma_devstat_t),
               cudaMemcpyDeviceToHost);
    int s = plasma->hstat->status;
    if (s != 0) {
        cudaMemset(plasma->dstat, 0, sizeof(plasma_devstat_t));
        cudaDeviceSynchronize();
    }
    return s;
}

/* R = B - A X, norms to the host arrays, returns conv() */
static int residual_check(plasma_context_t *plasma, plasma_enum_t uplo,
                          plasma_desc_t A, plasma_desc_t B, plasma_desc_t X,
                          plasma_desc_t R, double *d_norms, double *Rnorm,
                          double *Xnorm, double cte)
{
    int nrhs = B.n;
    double *d_x = d_norms, *d_r = d_norms + nrhs;
    plasma_cuda_residual(plasma->stream, plasma->dstat, uplo, A, B, X, R,
                         d_x, d_r);
    cudaMemcpyAsync(Xnorm, d_x, sizeof(double) * nrhs, cudaMemcpyDeviceToHost,
                    plasma->stream);
    cudaMemcpyAsync(Rnorm, d_r, sizeof(double) * nrhs, cudaMemcpyDeviceToHost,
                    plasma->stream);
    cudaStreamSynchronize(plasma->stream);
    return conv(Rnorm, Xnorm, nrhs, cte);
}

/*
 * The solver proper.  Returns through *iter and the sequence; fills `rep`
 * when not NULL.
 */
static void Xdsposv(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_desc_t B, plasma_desc_t X,
                    plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R,
                    double *Rnorm, double *Xnorm, int *iter,
                    plasma_sequence_t *sequence, plasma_request_t *request,
                    plasma_dsposv_info_t *rep)
{
    const double eps = DBL_EPSILON * 0.5;   /* LAPACK dlamch('E') */
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    int nrhs = B.n;
    *iter = 0;

    double *d_small = (double *)plasma_scratch(plasma, PLASMA_SLOT_SMALL,
                                               sizeof(double) * (2 * nrhs + 8));
    void *W32 = plasma_scratch(plasma, PLASMA_SLOT_WORK,
                               (size_t)As.mt * As.mb * As.mb * sizeof(float));
    if (d_small == NULL || W32 == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    double *d_anorm = d_small + 2 * nrhs;
    double *d_norms = d_small;

    cudaEvent_t e0 = NULL, e1 = NULL, e2 = NULL;
    if (rep) {
        memset(rep, 0, sizeof(*rep));
        rep->refinement = PlasmaRefineIR;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&e2);
        cudaEventRecord(e0, S);
    }

    int call = plasma_call_begin(plasma, sequence, request);
    double Anorm = 0.0;
    plasma_cuda_lansy_inf(S, st, uplo, A, d_anorm, NULL);
    cudaMemcpyAsync(&Anorm, d_anorm, sizeof(double), cudaMemcpyDeviceToHost, S);

    /* low-precision phase */
    int lowfail = 0;
    plasma_cuda_lag2s(S, st, call, B, Xs, PlasmaGeneral);
    plasma_cuda_lag2s(S, st, call, A, As, uplo);
    /* As may be padded to whole tiles: identity on the padding */
    if (As.m > A.m)
        plasma_cuda_set_diag(S, As, A.m, As.m, 1.0);
    int mode = plasma->mixed_mode == PlasmaFactorAuto ? PlasmaFactorTF32
                                                      : plasma->mixed_mode;
    if (rep) rep->factor_mode = mode;
    plasma_pXpotrf_mode(plasma, uplo, As, sequence, request, call, mode);
    if (take_status(plasma) != 0)
        lowfail = 1;
    if (rep)
        cudaEventRecord(e1, S);

    int converged = 0;
    if (!lowfail) {
        double cte = Anorm * eps * sqrt((double)A.n);
        plasma_cuda_trsm_sweep(S, st, uplo, PlasmaNoTrans, As, Xs, W32, 0);
        plasma_cuda_trsm_sweep(S, st, uplo, PlasmaTrans, As, Xs, W32, 1);
        plasma_cuda_slag2d(S, st, Xs, X);
        if (residual_check(plasma, uplo, A, B, X, R, d_norms, Rnorm, Xnorm, cte)) {
            *iter = 0;
            converged = 1;
        }
        for (int it = 0; !converged && it < ITERMAX; it++) {
            plasma_cuda_lag2s(S, st, call, R, Xs, PlasmaGeneral);
            plasma_cuda_trsm_sweep(S, st, uplo, PlasmaNoTrans, As, Xs, W32, 1);
            plasma_cuda_trsm_sweep(S, st, uplo, PlasmaTrans, As, Xs, W32, 1);
            plasma_cuda_slag2d(S, st, Xs, R);
            plasma_cuda_geadd(S, st, R, X);
            int ok = residual_check(plasma, uplo, A, B, X, R, d_norms, Rnorm,
                                    Xnorm, cte);
            if (take_status(plasma) != 0)
                break;       /* overflow of the residual in FP32 */
            if (ok) {
                *iter = it + 1;
                converged = 1;
            }
        }
    }
    if (rep) {
        cudaEventRecord(e2, S);
        cudaEventSynchronize(e2);
        float ms1 = 0, ms2 = 0;
        cudaEventElapsedTime(&ms1, e0, e1);
        cudaEventElapsedTime(&ms2, e1, e2);
        rep->factor_ms = ms1;
        rep->refine_ms = ms2;
        rep->ir_iterations = converged ? *iter : ITERMAX;
        rep->anorm = Anorm;
        rep->attempts = 1;
    }
    if (converged) {
        if (rep) {
            double be = 0.0;
            for (int j = 0; j < nrhs; j++) {
                double d = Anorm * Xnorm[j];
                double r = d > 0 ? Rnorm[j] / d : 0.0;
                if (r > be) be = r;
            }
            rep->backward_error = be;
            cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
        }
        return;
    }

    /* FP64 fallback (zcposv.c:524-538): factor A in place, X = B, solve */
    *iter = -ITERMAX - 1;
    call = plasma_call_begin(plasma, sequence, request);
    plasma_pXpotrf(plasma, uplo, A, sequence, request, call);
    plasma_cuda_lacpy(S, st, B, X);
    plasma_pXpotrs(plasma, uplo, A, X, sequence, request);
    if (rep) {
        rep->fallback_fp64 = 1;
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    }
}

static int check_descs(plasma_enum_t uplo, plasma_desc_t A, plasma_desc_t B,
                       plasma_desc_t X, plasma_desc_t As, plasma_desc_t Xs,
                       plasma_desc_t R, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    const plasma_desc_t *d[6] = {&A, &B, &X, &As, &Xs, &R};
    const char *names[6] = {"invalid A", "invalid B", "invalid X",
                            "invalid As", "invalid Xs", "invalid R"};
    for (int i = 0; i < 6; i++) {
        if (plasma_desc_check(*d[i]) != PlasmaSuccess) {
            plasma_error(names[i]);
            plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
            return 0;
        }
    }
    return 1;
}

void plasma_omp_dsposv(plasma_enum_t uplo,
                       plasma_desc_t A, plasma_desc_t B, plasma_desc_t X,
                       plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R,
                       double *W, double *Rnorm, double *Xnorm, int *iter,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    (void)W;
    *iter = 0;
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return;
    }
    if (!check_descs(uplo, A, B, X, As, Xs, R, sequence, request))
        return;
    if (A.n == 0 || B.n == 0)
        return;
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return;
    }
    if (sequence->status != PlasmaSuccess)
        return;
    Xdsposv(plasma, uplo, A, B, X, As, Xs, R, Rnorm, Xnorm, iter, sequence,
            request, NULL);
}

int plasma_dsposv_ex(plasma_enum_t uplo, int n, int nrhs,
                     double *pA, int lda, double *pB, int ldb,
                     double *pX, int ldx, int *iter,
                     plasma_dsposv_info_t *info)
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
    if (lda < imax(1, n)) {
        plasma_error("illegal value of lda");
        return -5;
    }
    if (ldb < imax(1, n)) {
        plasma_error("illegal value of ldb");
        return -7;
    }
    if (ldx < imax(1, n)) {
        plasma_error("illegal value of ldx");
        return -9;
    }
    *iter = 0;
    if (imin(n, nrhs) == 0)
        return PlasmaSuccess;
    if (plasma->device < 0)
        return PlasmaErrorEnvironment;

    if (plasma->tuning)
        plasma_tune_potrf(plasma, PlasmaRealFloat, n);
    int nb = plasma->nb;
    /* the low-precision operands are padded to whole tiles (identity on the
     * padding) so that the tensor-core kernels never see a ragged tile */
    int npad = ((n + nb - 1) / nb) * nb;

    plasma_desc_t A, B, X, R, As, Xs;
    memset(&A, 0, sizeof(A)); memset(&B, 0, sizeof(B));
    memset(&X, 0, sizeof(X)); memset(&R, 0, sizeof(R));
    memset(&As, 0, sizeof(As)); memset(&Xs, 0, sizeof(Xs));
    int retval;
    if ((retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, n,
                                             0, 0, n, n, &A)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &B)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &X)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &R)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealFloat, nb, nb, npad, npad,
                                             0, 0, npad, npad, &As)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealFloat, nb, nb, npad, nrhs,
                                             0, 0, npad, nrhs, &Xs)) != 0) {
        plasma_error("plasma_desc_general_create() failed");
        plasma_desc_destroy(&A); plasma_desc_destroy(&B);
        plasma_desc_destroy(&X); plasma_desc_destroy(&R);
        plasma_desc_destroy(&As); plasma_desc_destroy(&Xs);
        return retval;
    }
    double *Rnorm = (double *)malloc(sizeof(double) * nrhs);
    double *Xnorm = (double *)malloc(sizeof(double) * nrhs);

    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    /* only the uplo triangle of A is referenced */
    plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
    plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    if (sequence.status == PlasmaSuccess) {
        Xdsposv(plasma, uplo, A, B, X, As, Xs, R, Rnorm, Xnorm, iter,
                &sequence, &request, info);
    }
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(X, pX, ldx, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);

    plasma_desc_destroy(&A); plasma_desc_destroy(&B);
    plasma_desc_destroy(&X); plasma_desc_destroy(&R);
    plasma_desc_destroy(&As); plasma_desc_destroy(&Xs);
    free(Rnorm);
    free(Xnorm);
    return sequence.status;
}

int plasma_dsposv(plasma_enum_t uplo, int n, int nrhs,
                  double *pA, int lda, double *pB, int ldb,
                  double *pX, int ldx, int *iter)
{
    return plasma_dsposv_ex(uplo, n, nrhs, pA, lda, pB, ldb, pX, ldx, iter,
                            NULL);
}
