/*
 * dsgesv.c -- LU-based mixed-precision solver: plasma_dsgesv /
 * plasma_omp_dsgesv (compute/zcgesv.c:106-271 and :363-532), with the tile
 * LU with partial pivoting (compute/pzgetrf.c:37-232) and its solve
 * (compute/zgetrs.c, pzgeswp.c, pztrsm.c) that it runs in FP32 and, when
 * refinement fails, in FP64.
 *
 * Same interface and semantics as the reference: argument codes -1 (n),
 * -2 (nrhs), -4 (lda), -7 (ldb), -9 (ldx); iter = 0 on quick return; A and B
 * are not modified, X receives the solution, ipiv the pivots of the
 * factorization that produced it (1-based, LAPACK's convention); iter >= 0
 * refinement steps, or -31 when the FP64 factorization was used.  Stopping
 * rule of zcgesv.c:275-287: ||r_j||_inf <= ||x_j||_inf ||A||_inf eps sqrt(n)
 * for every column j, at most 30 steps.  As in LAPACK's dsgesv (and this
 * library's dsposv) an FP32 overflow of A or B, or a zero pivot of the FP32
 * factorization, goes straight to the FP64 factorization; info > 0 is the
 * first zero pivot of the FP64 factorization.
 *
 * The LU walk (plasma_pXgetrf), per tile column k on the context stream:
 *   PANEL(k)            k_lu_pivot / k_lu_update per column: pivots and
 *                       multipliers of tile column k
 *   LASWP(k)            the panel's interchanges on the other columns
 *   TRTRI(k)            inverses of the unit-lower and upper diagonal tile
 *   block row           A(k, k+1:) <- inv(L_kk) A(k, k+1:)   (GEMM on views)
 *   trailing update     A(k+1:, k+1:) -= A(k+1:, k) A(k, k+1:) (GEMM)
 * The reference defers the interchanges left of the panel to the end
 * (pzgetrf.c:196-228); they move values without arithmetic, so applying them
 * at once gives the same factors.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ITERMAX 30

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n);

/* Reads the device status after a stream sync and clears it. */
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

static plasma_view_t view(plasma_desc_t D, int r0, int c0)
{
    plasma_view_t v;
    memset(&v, 0, sizeof(v));
    v.D = D;
    v.r0 = r0;
    v.c0 = c0;
    return v;
}

/* Workspace of one LU of A: the inverses of all diagonal tiles (unit lower
 * and upper, nb x nb each, kept for the solves) and a block row. */
typedef struct {
    void *WL, *WU;
    plasma_desc_t Wd;      /* general nb x (mt*nb) view of WL ... */
    plasma_desc_t Wu;      /* ... and of WU                         */
    void *tmp;             /* nb x max(n, nrhs) block row            */
    size_t tmp_cols;
    void *parts;           /* per-CTA pivot candidates of the panel  */
    void *Wf, *Wb;         /* block inverses of the one-launch sweeps */
    int sweeps;            /* Wf, Wb hold the current factor's        */
    int *perm;             /* the interchanges as one permutation     */
    int permuted;          /* perm holds the current factor's         */
} lu_work_t;

static int lu_work(plasma_context_t *plasma, plasma_desc_t A, int ncols, lu_work_t *w)
{
    const size_t es = plasma_element_size(A.precision);
    const size_t nbsq = (size_t)A.mb * A.mb;
    const size_t wsw = (plasma_cuda_trsv_w_bytes(A) + 255) & ~(size_t)255;
    char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_WORK,
                                       2 * A.mt * nbsq * es + 2 * wsw +
                                           sizeof(int) * ((size_t)A.m + 8) + 256);
    const size_t cols = (size_t)(ncols > A.n ? ncols : A.n);
    void *tmp = plasma_scratch(plasma, PLASMA_SLOT_ADJOINT, (size_t)A.mb * cols * es + 256);
    void *parts = plasma_scratch(plasma, PLASMA_SLOT_MIXED, plasma_cuda_getrf_parts_bytes(A));
    if (buf == NULL || tmp == NULL || parts == NULL)
        return 0;
    w->parts = parts;
    w->WL = buf;
    w->WU = buf + A.mt * nbsq * es;
    w->Wf = buf + 2 * A.mt * nbsq * es;
    w->Wb = (char *)w->Wf + wsw;
    w->sweeps = 0;
    w->permuted = 0;
    w->perm = (int *)((char *)w->Wb + wsw);
    plasma_desc_general_init(A.precision, w->WL, A.mb, A.mb, A.mb, A.mt * A.mb, 0, 0,
                             A.mb, A.mt * A.mb, &w->Wd);
    plasma_desc_general_init(A.precision, w->WU, A.mb, A.mb, A.mb, A.mt * A.mb, 0, 0,
                             A.mb, A.mt * A.mb, &w->Wu);
    w->tmp = tmp;
    w->tmp_cols = cols;
    return 1;
}

/* the block row B(k, c0 : c0+N) <- W_k B(k, c0 : c0+N) through the block-row
 * buffer (W = Wd or Wu: the inverse of tile k at columns k*nb of it) */
static void apply_inverse(plasma_context_t *plasma, lu_work_t *w, plasma_desc_t W,
                          plasma_desc_t B, int k, int kb, int c0, int N)
{
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    plasma_desc_t T;
    plasma_desc_general_init(B.precision, w->tmp, B.mb, B.nb, B.mb, (int)w->tmp_cols, 0, 0,
                             kb, N, &T);
    plasma_cuda_copy_view(S, st, kb, N, view(B, k * B.mb, c0), view(T, 0, 0));
    plasma_cuda_gemm_view(S, st, kb, N, kb, 1.0, view(W, 0, k * W.mb), view(T, 0, 0), 0.0,
                          view(B, k * B.mb, c0), 0, 0);
}

/* LU with partial pivoting of the square general descriptor A in place;
 * dpiv (device, A.m entries) receives the pivots; the inverses of the
 * diagonal tiles stay in w for the solves.  A zero pivot records its info
 * in the device status and stops the walk (the later kernels see it). */
static void plasma_pXgetrf(plasma_context_t *plasma, plasma_desc_t A, int *dpiv,
                           lu_work_t *w, int call)
{
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    const int mt = A.mt < A.nt ? A.mt : A.nt;
    for (int k = 0; k < mt; k++) {
        const int kb = plasma_tile_nview(A, k);
        const int r0 = k * A.mb, c1 = r0 + kb;
        plasma_cuda_getrf_panel(S, st, call, A, k, dpiv, w->parts);
        plasma_cuda_laswp_skip(S, st, A, dpiv, r0, r0 + kb, 0, A.n, r0, c1);
        plasma_cuda_trtri_lu(S, st, A, k, k + 1, w->WL, w->WU);
        if (c1 < A.n) {
            if (!plasma_cuda_lu_rowsolve(S, st, A, k, w->WL))
                apply_inverse(plasma, w, w->Wd, A, k, kb, c1, A.n - c1);
            if (c1 < A.m && !plasma_cuda_lu_update(S, st, A, k))
                plasma_cuda_gemm_view(S, st, A.m - c1, A.n - c1, kb, -1.0, view(A, c1, r0),
                                      view(A, r0, c1), 1.0, view(A, c1, c1), 0, 0);
        }
    }
    /* the block inverses of the one-launch sweeps (one right-hand side) */
    w->sweeps = plasma_sweep_reserve(plasma, A) &&
                plasma_cuda_trtri_blocks_lu(S, st, A, w->Wf, w->Wb);
    w->permuted = plasma_cuda_lu_perm(S, st, dpiv, A.m, w->perm);
}

/* A X = B with the factor of plasma_pXgetrf (pivots dpiv, inverses in w):
 * the interchanges, then the unit-lower and the upper block sweeps. */
static void plasma_pXgetrs(plasma_context_t *plasma, plasma_desc_t A, const int *dpiv,
                           lu_work_t *w, plasma_desc_t B)
{
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    const int mt = A.mt, N = B.n;
    if (!(N == 1 && w->permuted && plasma_cuda_permute_vec(S, st, B, 0, w->perm, A.m)))
        plasma_cuda_laswp(S, st, B, dpiv, 0, A.m, 0, N);
    /* one right-hand side (a contiguous vector): the one-launch sweeps,
     * L y = P b (unit lower, forward), then U x = y (backward) */
    if (w->sweeps && N == 1 && B.gn == 1 && B.nt == 1) {
        plasma_sweep(plasma, PlasmaLower, 0, A, w->Wf, B.matrix);
        plasma_sweep(plasma, PlasmaUpper, 1, A, w->Wb, B.matrix);
        return;
    }
    for (int k = 0; k < mt; k++) {
        const int kb = plasma_tile_mview(A, k), r0 = k * A.mb, r1 = r0 + kb;
        apply_inverse(plasma, w, w->Wd, B, k, kb, 0, N);
        if (r1 < A.m)
            plasma_cuda_gemm_view(S, st, A.m - r1, N, kb, -1.0, view(A, r1, r0),
                                  view(B, r0, 0), 1.0, view(B, r1, 0), 0, 0);
    }
    for (int k = mt - 1; k >= 0; k--) {
        const int kb = plasma_tile_mview(A, k), r0 = k * A.mb;
        apply_inverse(plasma, w, w->Wu, B, k, kb, 0, N);
        if (r0 > 0)
            plasma_cuda_gemm_view(S, st, r0, N, kb, -1.0, view(A, 0, r0), view(B, r0, 0), 1.0,
                                  view(B, 0, 0), 0, 0);
    }
}

static int check_descs(plasma_desc_t A, plasma_desc_t B, plasma_desc_t X, plasma_desc_t As,
                       plasma_desc_t Xs, plasma_desc_t R)
{
    const plasma_desc_t *d[6] = {&A, &B, &X, &As, &Xs, &R};
    for (int i = 0; i < 6; i++)
        if (plasma_desc_check(*d[i]) != PlasmaSuccess || d[i]->type != PlasmaGeneral ||
            d[i]->i != 0 || d[i]->j != 0)
            return 0;
    if (A.precision != PlasmaRealDouble || B.precision != PlasmaRealDouble ||
        X.precision != PlasmaRealDouble || R.precision != PlasmaRealDouble ||
        As.precision != PlasmaRealFloat || Xs.precision != PlasmaRealFloat)
        return 0;
    if (A.m != A.n || As.m != A.m || As.n != A.n || B.m != A.m || X.m != A.m ||
        R.m != A.m || Xs.m != A.m || X.n != B.n || R.n != B.n || Xs.n != B.n)
        return 0;
    /* the same tiling everywhere (the solves and residuals mix them) */
    const plasma_desc_t *t[5] = {&B, &X, &As, &Xs, &R};
    for (int i = 0; i < 5; i++)
        if (t[i]->mb != A.mb || t[i]->nb != A.nb)
            return 0;
    return A.mb == A.nb;
}

/* R = B - A X; xn, rn (device) <- columnwise max |X|, |R|.  part: scratch
 * of the one-column product (plasma_cuda_gemv_part_bytes). */
static void residual(plasma_context_t *plasma, plasma_desc_t A, plasma_desc_t B,
                     plasma_desc_t X, plasma_desc_t R, double *xn, double *rn, double *part)
{
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    plasma_cuda_lacpy(S, st, B, R);
    if (B.n == 1 && X.gn == 1 && R.gn == 1)
        plasma_cuda_gemv_sub(S, st, A, X.matrix, R.matrix, part);
    else
        plasma_cuda_gemm_view(S, st, A.m, B.n, A.n, -1.0, view(A, 0, 0), view(X, 0, 0), 1.0,
                              view(R, 0, 0), 0, 0);
    plasma_cuda_colmax(S, st, X, xn);
    plasma_cuda_colmax(S, st, R, rn);
}

/* zcgesv.c conv() (Rnorm <= Xnorm * cte for every column), except that a
 * non-finite norm never counts as converged: the reference's form (fail
 * only if Rnorm > Xnorm * cte) passes a NaN residual, and an overflowed
 * iterate makes the bound infinite; such an iteration falls back to the
 * FP64 LU after its last step instead. */
static int converged(const double *rn, const double *xn, int nrhs, double cte)
{
    for (int j = 0; j < nrhs; j++)
        if (!isfinite(xn[j]) || !isfinite(rn[j]) || !(rn[j] <= xn[j] * cte))
            return 0;
    return 1;
}

void plasma_omp_dsgesv(plasma_desc_t A, int *ipiv, plasma_desc_t B, plasma_desc_t X,
                       plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R, double *work,
                       double *Rnorm, double *Xnorm, int *iter,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    (void)work;
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (sequence == NULL || request == NULL || iter == NULL || ipiv == NULL) {
        plasma_error("NULL sequence, request, iter or ipiv");
        return;
    }
    *iter = 0;
    if (!check_descs(A, B, X, As, Xs, R)) {
        plasma_error("invalid descriptors");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (A.n == 0 || B.n == 0)
        return;
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return;
    }
    if (A.mb > 512) {
        plasma_error("tile size not supported by the GPU kernels");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return;
    }
    if (sequence->status != PlasmaSuccess)
        return;
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    const int n = A.n, nrhs = B.n;
    const double eps = DBL_EPSILON * 0.5;     /* LAPACK dlamch('E') */

    double *dsmall = (double *)plasma_scratch(plasma, PLASMA_SLOT_SMALL,
                                              sizeof(double) * (2 * (size_t)nrhs + 8));
    int *dpiv = (int *)plasma_scratch(plasma, PLASMA_SLOT_SYMV, sizeof(int) * ((size_t)n + 8));
    double *part = (double *)plasma_scratch(plasma, PLASMA_SLOT_REFINE,
                                            plasma_cuda_gemv_part_bytes(A));
    double *hn = (double *)malloc(sizeof(double) * (2 * (size_t)nrhs + 1));
    lu_work_t w;
    if (dsmall == NULL || dpiv == NULL || part == NULL || hn == NULL ||
        !lu_work(plasma, A, nrhs, &w)) {
        free(hn);
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    double *d_anorm = dsmall, *d_xn = dsmall + 1, *d_rn = dsmall + 1 + nrhs;
    double *h_xn = hn, *h_rn = hn + nrhs;
    int call = plasma_call_begin(plasma, sequence, request);

    /* ||A||_inf, cte = ||A|| eps sqrt(n) (zcgesv.c:426-434) */
    double anorm = 0.0;
    plasma_cuda_lange_inf(S, st, A, d_anorm, part);
    cudaMemcpyAsync(&anorm, d_anorm, sizeof(double), cudaMemcpyDeviceToHost, S);
    int fallback = take_status(plasma) != 0;
    const double cte = anorm * eps * sqrt((double)n);

    /* FP32 copies of B and A (dlag2s: overflow -> the FP64 path) */
    if (!fallback) {
        plasma_cuda_lag2s(S, st, call, B, Xs, PlasmaGeneral);
        plasma_cuda_lag2s(S, st, call, A, As, PlasmaGeneral);
        fallback = take_status(plasma) != 0;
    }
    lu_work_t ws;
    if (!fallback && !lu_work(plasma, As, nrhs, &ws))
        fallback = 1;
    if (!fallback) {
        plasma_pXgetrf(plasma, As, dpiv, &ws, call);
        fallback = take_status(plasma) != 0;       /* a zero FP32 pivot */
    }
    int done = 0;
    if (!fallback) {
        plasma_pXgetrs(plasma, As, dpiv, &ws, Xs);
        plasma_cuda_slag2d(S, st, Xs, X);
        residual(plasma, A, B, X, R, d_xn, d_rn, part);
        cudaMemcpyAsync(hn, d_xn, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, S);
        cudaStreamSynchronize(S);
        done = converged(h_rn, h_xn, nrhs, cte);
        for (int it = 0; !done && it < ITERMAX; it++) {
            plasma_cuda_lag2s(S, st, call, R, Xs, PlasmaGeneral);
            if (take_status(plasma) != 0)
                break;                                   /* R overflows FP32 */
            plasma_pXgetrs(plasma, As, dpiv, &ws, Xs);
            plasma_cuda_slag2d(S, st, Xs, R);
            plasma_cuda_geadd(S, st, R, X);
            residual(plasma, A, B, X, R, d_xn, d_rn, part);
            cudaMemcpyAsync(hn, d_xn, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, S);
            cudaStreamSynchronize(S);
            done = converged(h_rn, h_xn, nrhs, cte);
            if (done)
                *iter = it + 1;
        }
    }
    if (!done) {
        /* FP64 (zcgesv.c:511-531): factor A in place, X = B, solve */
        *iter = -ITERMAX - 1;
        if (!lu_work(plasma, A, nrhs, &w)) {
            free(hn);
            plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
            return;
        }
        plasma_pXgetrf(plasma, A, dpiv, &w, call);
        plasma_cuda_lacpy(S, st, B, X);
        plasma_pXgetrs(plasma, A, dpiv, &w, X);
    }
    if (Xnorm != NULL && done)
        memcpy(Xnorm, h_xn, sizeof(double) * nrhs);
    if (Rnorm != NULL && done)
        memcpy(Rnorm, h_rn, sizeof(double) * nrhs);
    cudaMemcpyAsync(ipiv, dpiv, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, S);
    cudaStreamSynchronize(S);
    free(hn);
}

int plasma_dsgesv(int n, int nrhs, double *pA, int lda, int *ipiv, double *pB, int ldb,
                  double *pX, int ldx, int *iter)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    if (n < 0) {
        plasma_error("illegal value of n");
        return -1;
    }
    if (nrhs < 0) {
        plasma_error("illegal value of nrhs");
        return -2;
    }
    if (lda < imax(1, n)) {
        plasma_error("illegal value of lda");
        return -4;
    }
    if (ldb < imax(1, n)) {
        plasma_error("illegal value of ldb");
        return -7;
    }
    if (ldx < imax(1, n)) {
        plasma_error("illegal value of ldx");
        return -9;
    }
    if (iter != NULL)
        *iter = 0;
    if (imin(n, nrhs) == 0)
        return PlasmaSuccess;
    if (ipiv == NULL || iter == NULL)
        return PlasmaErrorIllegalValue;
    if (plasma->device < 0)
        return PlasmaErrorEnvironment;
    /* tuned: 64-wide tiles when the FP32 LU's panels fit the one-launch
     * cluster panel (the panel's column chain is the LU's critical path;
     * wider tiles only lengthen it), else the Cholesky table's size */
    int nb = plasma->nb;
    if (plasma->tuning) {
        if (n <= plasma_cuda_getrf_cluster_rows(PlasmaRealFloat)) {
            nb = 64;
        } else {
            plasma_tune_potrf(plasma, PlasmaRealFloat, n);
            nb = plasma->nb;
        }
    }

    plasma_desc_t A, As, B, X, Xs, R;
    int rc = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, PlasmaRealDouble, PlasmaGeneral, nb,
                              n, n, &A);
    if (rc == PlasmaSuccess)
        rc = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_AS, PlasmaRealFloat, PlasmaGeneral, nb,
                              n, n, &As);
    if (rc != PlasmaSuccess)
        return rc;
    plasma_desc_t *rhs[4] = {&B, &X, &R, &Xs};
    int made = 0;
    for (; made < 4 && rc == PlasmaSuccess; made++)
        rc = plasma_desc_general_create(made == 3 ? PlasmaRealFloat : PlasmaRealDouble, nb, nb,
                                        n, nrhs, 0, 0, n, nrhs, rhs[made]);
    if (rc != PlasmaSuccess) {
        for (int i = 0; i < made - 1; i++)
            plasma_desc_destroy(rhs[i]);
        return rc;
    }
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    plasma_omp_Xlapack2desc(pA, lda, A, PlasmaGeneral, &sequence, &request);
    plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    plasma_omp_dsgesv(A, ipiv, B, X, As, Xs, R, NULL, NULL, NULL, iter, &sequence, &request);
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(X, pX, ldx, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);
    for (int i = 0; i < 4; i++)
        plasma_desc_destroy(rhs[i]);
    return sequence.status;
}
