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
 * Failures, as the reference: in its own configuration (FP32 factor,
 * classical IR -- the defaults) a failed FP32 factorisation fails the call
 * with that factorisation's info (the first non-positive leading minor of
 * the FP32 matrix), and an FP32 overflow in a conversion (of A, B or a
 * residual) fails it with info = 1; iter is then -31 and X is not written.
 * The reference gets there by cancelling every later task of the sequence
 * (each core task tests sequence->status first), so that its FP64 fallback
 * never runs; its iter in that case is read from buffers no task filled,
 * and -31 is what it returns in practice.  The reference's tester checks
 * only info (test/test_zcposv.c:181-192).  The extended configurations
 * (TF32 / BF16 / Auto factors, GMRES-IR or the automatic scheme) retry a
 * failed factorisation scaled and shifted and then fall back to FP64, as
 * LAPACK's dsposv does on an FP32 failure.
 *
 * Deliberate differences (also listed in the design notes):
 *  - Only the uplo triangle of A is converted (the reference converts the full
 *    general matrix, with a "TODO: need zlat2c" note at zcposv.c:447, so an
 *    FP32 overflow in the triangle it never reads also gives info = 1), and
 *    into the LOWER triangle of As whatever uplo is (transposed tiles for
 *    uplo = Upper), so that the FP32 factor is always the lower one.
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

/* ------------------------------------------------------------------------
 * Refinement on contiguous vectors, one right-hand side at a time.
 * ---------------------------------------------------------------------- */
#define GMRES_RESTART 40
#define GMRES_TOL 1e-6

typedef struct {
    plasma_context_t *plasma;
    plasma_enum_t uplo;               /* stored triangle of A            */
    plasma_enum_t uplo_s;             /* stored triangle of As (factor)  */
    plasma_desc_t A, As;
    const void *W32;
    int call;
    size_t n, npad;
    double *b, *x, *r, *w, *z, *V;   /* FP64 vectors, V: (m+1) x n basis */
    const double *dscale;             /* D^{-1} of a scaled factor, or NULL */
    int fast;                         /* one-launch sweeps (else tile sweeps) */
    float *ws;                        /* FP32 work vector (npad)        */
    double *dh, *dnorm, *dwork;       /* small device buffers           */
    double *symv_work;
    int gmres_iters;
} refine_t;

/* out = M^{-1} in with M the low-precision factorisation of A */
static void precond(refine_t *R, const double *in, double *out)
{
    cudaStream_t S = R->plasma->stream;
    /* M = D^{-1} L L^T D^{-1} when the factor is of the scaled matrix
     * D A D (+ shift): M^{-1} v = D (L L^T)^{-1} D v */
    plasma_cuda_d2s(S, in, R->dscale, R->ws, R->n, R->npad, R->plasma->dstat, R->call);
    if (R->fast) {
        plasma_sweep(R->plasma, R->uplo_s, 0, R->As, R->W32, R->ws);
        plasma_sweep(R->plasma, R->uplo_s, 1, R->As, R->W32, R->ws);
    } else {
        /* the vector viewed as an npad x 1 tile descriptor */
        plasma_desc_t V;
        plasma_desc_general_init(PlasmaRealFloat, R->ws, R->As.mb, R->As.nb,
                                 (int)R->npad, 1, 0, 0, (int)R->npad, 1, &V);
        plasma_cuda_trsm_sweep(S, R->plasma->dstat, R->uplo_s, PlasmaNoTrans,
                               R->As, V, (void *)R->W32, 1);
        plasma_cuda_trsm_sweep(S, R->plasma->dstat, R->uplo_s, PlasmaTrans,
                               R->As, V, (void *)R->W32, 1);
    }
    plasma_cuda_s2d(S, R->ws, R->dscale, out, R->n);
}

/* r = b - A x, returns the max norms of x and r through the host pointers */
static void residual_vec(refine_t *R, double *xn, double *rn)
{
    cudaStream_t S = R->plasma->stream;
    plasma_cuda_symv(S, R->plasma->dstat, R->uplo, R->A, R->x, R->b, R->r,
                     R->dnorm, R->dnorm + 1, R->symv_work);
    double h[2];
    cudaMemcpyAsync(h, R->dnorm, sizeof(h), cudaMemcpyDeviceToHost, S);
    cudaStreamSynchronize(S);
    *xn = h[0];
    *rn = h[1];
}

static double dot_host(refine_t *R, const double *a, const double *b)
{
    cudaStream_t S = R->plasma->stream;
    double v;
    plasma_cuda_dots(S, a, 0, 1, b, R->n, R->dh, R->dwork);
    cudaMemcpyAsync(&v, R->dh, sizeof(double), cudaMemcpyDeviceToHost, S);
    cudaStreamSynchronize(S);
    return v;
}

/* One GMRES solve of M^{-1} A d = M^{-1} r (restart length GMRES_RESTART,
 * relative tolerance GMRES_TOL), x += d.  Returns the inner iterations. */
static int gmres_correction(refine_t *R)
{
    cudaStream_t S = R->plasma->stream;
    const size_t n = R->n;
    const int m = GMRES_RESTART;
    double H[GMRES_RESTART + 1][GMRES_RESTART];
    double cs[GMRES_RESTART], sn[GMRES_RESTART], g[GMRES_RESTART + 1];
    double hcol[GMRES_RESTART + 1], hcol2[GMRES_RESTART + 1], y[GMRES_RESTART];
    double gtrace[GMRES_RESTART];      /* |g_{j+1}|, the residual after step j */

    precond(R, R->r, R->z);
    double beta = sqrt(dot_host(R, R->z, R->z));
    if (!(beta > 0.0))
        return 0;
    plasma_cuda_axpby(S, 1.0 / beta, R->z, R->V, n, 0);
    for (int i = 0; i <= m; i++) g[i] = 0.0;
    g[0] = beta;
    int k = 0;
    for (int j = 0; j < m; j++) {
        double *vj = R->V + (size_t)j * n;
        /* w = M^{-1} A v_j */
        plasma_cuda_symv(S, R->plasma->dstat, R->uplo, R->A, vj, NULL, R->z,
                         NULL, NULL, R->symv_work);
        precond(R, R->z, R->w);
        /* classical Gram-Schmidt, twice */
        plasma_cuda_dots(S, R->V, n, j + 1, R->w, n, R->dh, R->dwork);
        plasma_cuda_sub_combo(S, R->V, n, j + 1, R->dh, R->w, n);
        cudaMemcpyAsync(hcol, R->dh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, S);
        plasma_cuda_dots(S, R->V, n, j + 1, R->w, n, R->dh, R->dwork);
        plasma_cuda_sub_combo(S, R->V, n, j + 1, R->dh, R->w, n);
        cudaMemcpyAsync(hcol2, R->dh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, S);
        cudaStreamSynchronize(S);
        for (int i = 0; i <= j; i++) hcol[i] += hcol2[i];
        double hn = sqrt(dot_host(R, R->w, R->w));
        hcol[j + 1] = hn;
        if (hn > 0.0)
            plasma_cuda_axpby(S, 1.0 / hn, R->w, R->V + (size_t)(j + 1) * n, n, 0);
        /* Givens rotations on the new Hessenberg column */
        for (int i = 0; i < j; i++) {
            double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
            hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
            hcol[i] = t;
        }
        double a = hcol[j], bb = hcol[j + 1];
        double rr = hypot(a, bb);
        cs[j] = rr > 0.0 ? a / rr : 1.0;
        sn[j] = rr > 0.0 ? bb / rr : 0.0;
        hcol[j] = rr;
        hcol[j + 1] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        for (int i = 0; i <= j; i++) H[i][j] = hcol[i];
        k = j + 1;
        R->gmres_iters++;
        if (fabs(g[j + 1]) <= GMRES_TOL * beta || !(hn > 0.0))
            break;
        /* a stagnating Krylov residual (less than 2x over the last 20
         * steps): the preconditioner is too weak, end this solve early */
        if (j >= 20 && fabs(g[j + 1]) > 0.5 * gtrace[j - 20])
            break;
        gtrace[j] = fabs(g[j + 1]);
    }
    /* back substitution H(0:k,0:k) y = g(0:k) */
    for (int i = k - 1; i >= 0; i--) {
        double t = g[i];
        for (int l = i + 1; l < k; l++) t -= H[i][l] * y[l];
        y[i] = H[i][i] != 0.0 ? t / H[i][i] : 0.0;
    }
    cudaMemcpyAsync(R->dh, y, sizeof(double) * k, cudaMemcpyHostToDevice, S);
    plasma_cuda_combo(S, R->V, n, k, R->dh, R->x, n, 1);
    return k;
}

/* Solves for the current b: initial x = M^{-1} b, then refinement until the
 * reference stopping rule holds.  Returns the number of refinement steps, or
 * -1 when it did not converge within ITERMAX. */
static int refine_column(refine_t *R, int scheme, double cte, int give_up,
                         double *xn_out, double *rn_out, int *used_gmres, int *status)
{
    precond(R, R->b, R->x);
    double prev = INFINITY;
    int gm = scheme == PlasmaRefineGMRES;
    int stalls = 0;
    for (int it = 0; it <= ITERMAX; it++) {
        double xn, rn;
        residual_vec(R, &xn, &rn);
        *xn_out = xn;
        *rn_out = rn;
        if ((*status = take_status(R->plasma)) != 0)
            return -1;                     /* FP32 overflow in a conversion */
        /* stopping rule of the reference's conv(), zcposv.c:275-287, except
         * that a non-finite norm never counts as converged (the reference's
         * form passes a NaN residual, and an overflowed iterate makes the
         * bound infinite) */
        if (isfinite(xn) && isfinite(rn) && rn <= xn * cte)
            return it;
        if (it == ITERMAX)
            break;
        /* give_up (the extended configurations): a factor that no longer
         * contracts the residual -- IR: less than 2x per step, GMRES-IR: less
         * than 10x per restarted solve, twice in a row, or a growing
         * residual -- is abandoned for the next attempt instead of running
         * out the 30 steps.  The reference's configuration always runs
         * them (zcposv.c:485-518). */
        /* automatic scheme: switch to GMRES-IR when IR stops contracting
         * (before any giving up: GMRES gets its chance first) */
        if (scheme == PlasmaRefineAuto && !gm && it > 0 && rn > 0.5 * prev) {
            gm = 1;
            stalls = 0;
        } else if (give_up && it > 0) {
            const double need = gm ? 0.1 : 0.5;
            stalls = (rn > need * prev) ? stalls + 1 : 0;
            if (!(rn < prev) || stalls >= 2)
                return -1;
        }
        prev = rn;
        if (gm) {
            *used_gmres = 1;
            gmres_correction(R);
        } else {
            precond(R, R->r, R->z);
            plasma_cuda_axpby(R->plasma->stream, 1.0, R->z, R->x, R->n, 1);
        }
    }
    return -1;
}

/* The caller's lower-stored matrix, converted inside the solve: from the
 * host, with the upload overlapping the factorization; from the device, in
 * one pass to the FP64 tiles of A and the FP32 tiles of As. */
typedef struct {
    const double *pA;
    int lda;
    int on_device;
    int pageable;        /* host memory that is not page-locked */
} upload_t;

/* Tile-column groups that each hold about the same share of the lower
 * triangle (up to PLASMA_MAX_GROUPS of them, so the first ones are narrow
 * and the last ones wide): the right-looking update of a column needs every
 * panel before it, so most of the update work sits in the last columns,
 * and fine groups let it start as early as the bus allows. */
static int column_groups(int nt, int *gstart)
{
    const int ng_max = nt < PLASMA_MAX_GROUPS ? nt : PLASMA_MAX_GROUPS;
    const double total = 0.5 * (double)nt * (nt + 1);
    int ng = 0;
    double acc = 0.0;
    gstart[0] = 0;
    for (int j = 0; j < nt; j++) {
        acc += nt - j;                      /* tiles of column j */
        if ((ng < ng_max - 1 && acc >= total * (ng + 1) / ng_max) || j == nt - 1)
            gstart[++ng] = j + 1;
    }
    return ng;
}

/* The first attempt of the FP32 path for a host matrix: its lower triangle
 * goes up on the copy stream one group of tile columns at a time (one
 * cudaMemcpy2DAsync per tile column, from the diagonal down), each group is
 * converted to the FP64 tiles of A and the FP32 tiles of As as soon as it
 * is in, and the factorization of As runs on the groups already in place
 * (plasma_pXpotrf_arrivals).  ||A||_inf follows the last group on the copy
 * stream.  Page-locked host memory is copied directly; pageable memory goes
 * through the staging slots (plasma_stage_copy), and both overlap the
 * kernels. */
static void upload_and_factor(plasma_context_t *plasma, const upload_t *up,
                              plasma_desc_t A, plasma_desc_t As, double *d_anorm,
                              double *symv_work, int call, int mode,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    cudaStream_t S = plasma->stream;
    cudaStream_t cp = plasma->aux[PLASMA_STREAM_COPY];
    plasma_devstat_t *st = plasma->dstat;
    const int n = A.m, nb = A.nb;
    /* every slot the factorization uses is sized before the first copy: a
     * slot that grows waits for all streams, the copy stream included */
    plasma_pXpotrf_reserve(plasma, PlasmaLower, As, mode, 1);
    double *stage = (double *)plasma_scratch(plasma, PLASMA_SLOT_STAGING,
                                             (size_t)n * (size_t)n * sizeof(double));
    if (stage == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    int gstart[PLASMA_MAX_GROUPS + 1];
    const int ng = column_groups(A.nt, gstart);
    /* the copies start after everything enqueued so far (the zeroed tile
     * storage, the right-hand side) */
    cudaEventRecord(plasma->ev[4], S);
    cudaStreamWaitEvent(cp, plasma->ev[4], 0);
    if (up->pageable)
        plasma_stage_begin(plasma, S);
    for (int g = 0; g < ng; g++) {
        for (int j = gstart[g]; j < gstart[g + 1]; j++) {
            const int c0 = j * nb;
            const int w = n - c0 < nb ? n - c0 : nb;
            double *dst = stage + (size_t)c0 * n + c0;
            const double *src = up->pA + (size_t)c0 * up->lda + c0;
            const size_t ldd = (size_t)n * sizeof(double), lds = (size_t)up->lda * sizeof(double);
            const size_t bytes = (size_t)(n - c0) * sizeof(double);
            if (up->pageable)
                plasma_stage_copy(plasma, dst, ldd, src, lds, bytes, (size_t)w,
                                  cudaMemcpyHostToDevice);
            else
                cudaMemcpy2DAsync(dst, ldd, src, lds, bytes, (size_t)w, cudaMemcpyHostToDevice,
                                  cp);
        }
        if (up->pageable)
            plasma_stage_join(plasma, cp);       /* the group's columns are in */
        plasma_cuda_upload_cols(cp, st, call, A, As, stage, n, gstart[g], gstart[g + 1]);
        cudaEventRecord(plasma->ev_group[g], cp);
    }
    plasma_cuda_lansy_inf(cp, plasma->dquiet, PlasmaLower, A, d_anorm, symv_work);
    cudaEventRecord(plasma->ev[5], cp);
    plasma_pXpotrf_arrivals(plasma, PlasmaLower, As, sequence, request, call, mode, ng,
                            gstart, plasma->ev_group);
    cudaStreamWaitEvent(S, plasma->ev[5], 0);
}

/*
 * The solver proper.  Returns through *iter and the sequence; fills `rep`
 * when not NULL.  up != NULL: A (lower) is still on the host and comes up
 * during the first factorization (upload_and_factor).
 */
static void Xdsposv(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_desc_t B, plasma_desc_t X,
                    plasma_desc_t As, plasma_desc_t Xs, plasma_desc_t R,
                    double *Rnorm, double *Xnorm, int *iter,
                    plasma_sequence_t *sequence, plasma_request_t *request,
                    plasma_dsposv_info_t *rep, const upload_t *up)
{
    const double eps = DBL_EPSILON * 0.5;   /* LAPACK dlamch('E') */
    cudaStream_t S = plasma->stream;
    plasma_devstat_t *st = plasma->dstat;
    int nrhs = B.n;
    *iter = 0;
    /* The FP32 copy and its factor live in LOWER storage whatever triangle
     * the caller stores A in (an upper-stored A is converted by transposed
     * tiles): the tensor-core trailing update of the factorisation runs on
     * lower tiles.  Only an As that is itself a packed upper triangle keeps
     * the upper factor.  A keeps the caller's triangle (norm, residual and
     * the FP64 fallback read it there). */
    const plasma_enum_t uplo_s = As.type == PlasmaUpper ? PlasmaUpper : PlasmaLower;

    /* the small device buffers at their full size from the start, so that
     * the slot never grows (and moves) during the solve */
    double *d_small = (double *)plasma_scratch(plasma, PLASMA_SLOT_SMALL,
                                               sizeof(double) * (2 * nrhs + 8) +
                                               sizeof(double) * (GMRES_RESTART + 8) +
                                               plasma_cuda_dots_work(GMRES_RESTART + 2));
    const int fast_sweep = plasma_sweep_reserve(plasma, As);
    size_t wtiles = (size_t)As.mt * As.mb * As.mb * sizeof(float);
    size_t wblocks = plasma_cuda_trsv_w_bytes(As);
    void *W32 = plasma_scratch(plasma, PLASMA_SLOT_WORK,
                               wtiles > wblocks ? wtiles : wblocks);
    if (d_small == NULL || W32 == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    double *d_anorm = d_small + 2 * nrhs;

    cudaEvent_t e0 = NULL, e1 = NULL, e2 = NULL;
    if (rep) {
        memset(rep, 0, sizeof(*rep));
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&e2);
        cudaEventRecord(e0, S);
    }

    int call = plasma_call_begin(plasma, sequence, request);
    double Anorm = 0.0;
    double *sw = (double *)plasma_scratch(plasma, PLASMA_SLOT_SYMV,
                                          plasma_cuda_symv_work(A));
    if (up != NULL && up->on_device)
        plasma_cuda_upload_cols(S, st, call, A, As, up->pA, up->lda, 0, A.nt);
    if (up == NULL || up->on_device) {
        plasma_cuda_lansy_inf(S, st, uplo, A, d_anorm, sw);
        cudaMemcpyAsync(&Anorm, d_anorm, sizeof(double), cudaMemcpyDeviceToHost, S);
    }

    /* ------------------------------------------------------------------
     * Low-precision phase.  An attempt = convert A, optionally scale it to
     * unit diagonal and shift it by c*u (Higham & Pranesh 2019), factor it
     * with the attempt's product precision, refine.  The reference's FP32
     * mode makes one unscaled attempt; TF32 / BF16 retry once scaled and
     * shifted when the factorisation breaks down; Auto escalates
     * BF16 -> TF32 -> FP32.  Whatever fails ends in the FP64 path below.
     * ---------------------------------------------------------------- */
    /* scaled: 0 = as is; c > 0 = unit diagonal and a shift of c*u */
    typedef struct { int mode; double scaled; } attempt_t;
    attempt_t plan[10];
    int nplan = 0;
    const int cfg = plasma->mixed_mode;
    if (cfg == PlasmaFactorAuto) {
        plan[nplan++] = (attempt_t){PlasmaFactorBF16, 0};
        plan[nplan++] = (attempt_t){PlasmaFactorBF16, 4};
        plan[nplan++] = (attempt_t){PlasmaFactorTF32, 4};
        plan[nplan++] = (attempt_t){PlasmaFactorFP32, 0};
        for (double c = 4; c <= 16384; c *= 16)
            plan[nplan++] = (attempt_t){PlasmaFactorFP32, c};
    } else if (cfg == PlasmaFactorFP32) {
        plan[nplan++] = (attempt_t){PlasmaFactorFP32, 0};
        /* a breakdown is retried with shifts of 4u, 64u, 1024u, 16384u:
         * the factorization's rounding error grows with the order and the
         * norm of the scaled matrix, and GMRES-IR tolerates a shifted
         * preconditioner */
        if (plasma->refinement != PlasmaRefineIR)
            for (double c = 4; c <= 16384; c *= 16)
                plan[nplan++] = (attempt_t){PlasmaFactorFP32, c};
    } else {
        /* TF32 / BF16 first, then FP32: a factor too coarse for the
         * matrix's condition escalates to FP32 before the FP64 fallback */
        plan[nplan++] = (attempt_t){cfg, 0};
        plan[nplan++] = (attempt_t){cfg, 4};
        plan[nplan++] = (attempt_t){PlasmaFactorFP32, 0};
        for (double c = 4; c <= 16384; c *= 16)
            plan[nplan++] = (attempt_t){PlasmaFactorFP32, c};
    }
    const int scheme = plasma->refinement;
    /* the reference's configuration keeps the reference's failure semantics */
    const int ref_failure = cfg == PlasmaFactorFP32 && scheme == PlasmaRefineIR;
    const size_t n = (size_t)A.m, npad = (size_t)As.m;
    const int mres = GMRES_RESTART;
    double cte = 0.0;
    int converged = 0, used_gmres = 0, gm_iters = 0, attempts = 0;
    int factor_failed = 0, fstatus = 0, last = 0;

    plasma_cuda_lag2s(S, st, call, B, Xs, PlasmaGeneral);
    size_t need = sizeof(double) * (size_t)n * (6 + mres + 1) +
                  sizeof(double) * npad + sizeof(float) * npad + 4096;
    char *wk = (char *)plasma_scratch(plasma, PLASMA_SLOT_REFINE, need);
    double *small = d_small;
    if (wk == NULL || small == NULL || sw == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    refine_t RF;
    memset(&RF, 0, sizeof(RF));
    RF.plasma = plasma;
    RF.uplo = uplo;
    RF.uplo_s = uplo_s;
    RF.A = A;
    RF.As = As;
    RF.W32 = W32;
    RF.fast = fast_sweep;
    RF.call = call;
    RF.n = n;
    RF.npad = npad;
    double *vp = (double *)wk;
    RF.b = vp; vp += n;
    RF.x = vp; vp += n;
    RF.r = vp; vp += n;
    RF.w = vp; vp += n;
    RF.z = vp; vp += n;
    RF.V = vp; vp += (size_t)n * (mres + 1);
    double *dvec = vp; vp += npad;
    RF.ws = (float *)vp;
    RF.dnorm = small + 2 * nrhs + 2;
    RF.dh = RF.dnorm + 4;
    RF.dwork = RF.dh + mres + 4;
    RF.symv_work = sw;

    for (int a = 0; a < nplan && !converged; a++) {
        const int mode = plan[a].mode;
        /* a scaled (and shifted) factor of the same precision follows one
         * that broke down, and, under GMRES-IR or the automatic scheme, an
         * unscaled one that did not refine (equilibration can make the
         * factor a good preconditioner, not a contraction for plain IR);
         * larger shifts only follow a scaled factorization that broke down */
        if (a > 0 && plan[a].scaled > 0 && plan[last].mode == mode && !factor_failed &&
            (plan[last].scaled > 0 || scheme == PlasmaRefineIR))
            continue;
        last = a;
        attempts++;
        if (rep) rep->factor_mode = mode;
        if (a > 0 && rep) cudaEventRecord(e0, S);
        /* As may be padded to whole tiles: identity on the padding */
        if (As.m > A.m)
            plasma_cuda_set_diag(S, As, A.m, As.m, 1.0);
        RF.dscale = NULL;
        if (a == 0 && up != NULL && !up->on_device) {
            upload_and_factor(plasma, up, A, As, d_anorm, sw, call, mode, sequence, request);
            cudaMemcpyAsync(&Anorm, d_anorm, sizeof(double), cudaMemcpyDeviceToHost, S);
            fstatus = take_status(plasma);
            factor_failed = fstatus != 0;
            if (rep)
                cudaEventRecord(e1, S);
            if (factor_failed && ref_failure)
                goto failed;
            if (factor_failed)
                continue;
            goto factored;
        }
        /* (a device A of the first attempt was converted with As above) */
        if (a > 0 || up == NULL) {
            if (uplo_s == uplo)
                plasma_cuda_lag2s(S, st, call, A, As, uplo);
            else
                plasma_cuda_lag2s_upper_to_lower(S, st, call, A, As);
        }
        if (plan[a].scaled > 0) {
            /* unit diagonal, then + c u I with u the unit roundoff of the
             * products and c from the plan */
            double u = mode == PlasmaFactorBF16 ? 0x1p-8 :
                       mode == PlasmaFactorTF32 ? 0x1p-11 : 0x1p-24;
            plasma_cuda_diag_rsqrt(S, A, dvec, n, npad);
            plasma_cuda_scale_shift(S, As, uplo_s, dvec, (float)(plan[a].scaled * u));
            RF.dscale = dvec;
        }
        plasma_pXpotrf_mode(plasma, uplo_s, As, sequence, request, call, mode);
        fstatus = take_status(plasma);
        factor_failed = fstatus != 0;
        if (rep)
            cudaEventRecord(e1, S);
        if (factor_failed && ref_failure)
            goto failed;
        if (factor_failed)
            continue;
    factored:
        cte = Anorm * eps * sqrt((double)A.n);
        /* inverses of the diagonal blocks of the factor, used by every sweep */
        if (fast_sweep)
            plasma_cuda_trtri_blocks(S, st, uplo_s, As, W32);
        else
            plasma_cuda_trtri_tiles(S, st, uplo_s, As, W32);
        converged = 1;
        int itmax = 0;
        for (int j = 0; j < nrhs; j++) {
            plasma_cuda_column(S, B, j, RF.b, 1);
            double xn = 0, rn = 0;
            int cstat = 0;
            int it = refine_column(&RF, scheme, cte, !ref_failure, &xn, &rn, &used_gmres,
                                   &cstat);
            Xnorm[j] = xn;
            Rnorm[j] = rn;
            if (cstat != 0 && ref_failure) {
                fstatus = cstat;
                goto failed;
            }
            if (it < 0) {
                converged = 0;
                break;
            }
            if (it > itmax) itmax = it;
            plasma_cuda_column(S, X, j, RF.x, 0);
        }
        if (converged)
            *iter = itmax;
    }
    gm_iters = RF.gmres_iters;
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
        rep->attempts = attempts;
        rep->refinement = used_gmres ? PlasmaRefineGMRES : PlasmaRefineIR;
        rep->gmres_iterations = gm_iters;
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
    return;

failed:
    /* the reference's cancelled sequence: its info, iter = -31, no solve */
    *iter = -ITERMAX - 1;
    plasma_request_fail(sequence, request, fstatus);
    if (rep) {
        rep->attempts = attempts;
        rep->anorm = Anorm;
        cudaEventRecord(e2, S);
        cudaEventSynchronize(e2);
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
    /* a packed triangle must hold the triangle the solve reads: A the
     * uplo one; As lower (any uplo) or, for uplo = Upper only, upper */
    if ((A.type == PlasmaLower || A.type == PlasmaUpper) && A.type != uplo) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (As.type == PlasmaUpper && uplo != PlasmaUpper) {
        plasma_error("invalid As");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
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
            request, NULL, NULL);
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
    /* A: the packed uplo triangle, As: the packed lower triangle (half the
     * memory of general storage; every kernel of the solve reads the stored
     * triangle only), held in
     * scratch slots that the context keeps between calls, so a solve
     * neither allocates nor frees its two large tile copies; zeroed on the
     * stream (the padding of As and the unreferenced halves of diagonal
     * tiles must hold finite values) */
    if ((retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_A, PlasmaRealDouble, uplo, nb, n,
                                   n, &A)) != 0 ||
        (retval = plasma_desc_kept(plasma, PLASMA_SLOT_DESC_AS, PlasmaRealFloat, PlasmaLower,
                                   nb, npad, npad, &As)) != 0)
        return retval;
    if ((retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &B)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &X)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealDouble, nb, nb, n, nrhs,
                                             0, 0, n, nrhs, &R)) != 0 ||
        (retval = plasma_desc_general_create(PlasmaRealFloat, nb, nb, npad, nrhs,
                                             0, 0, npad, nrhs, &Xs)) != 0) {
        plasma_error("plasma_desc_general_create() failed");
        plasma_desc_destroy(&B);
        plasma_desc_destroy(&X); plasma_desc_destroy(&R);
        plasma_desc_destroy(&Xs);
        return retval;
    }
    double *Rnorm = (double *)malloc(sizeof(double) * nrhs);
    double *Xnorm = (double *)malloc(sizeof(double) * nrhs);

    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    /* only the uplo triangle of A is referenced; a lower triangle on the
     * host goes up while the factorization runs (PLASMA_PIPELINE_UPLOAD=0
     * uploads it first) */
    static int pipeline_env = -1;
    if (pipeline_env < 0) {
        const char *e = getenv("PLASMA_PIPELINE_UPLOAD");
        pipeline_env = e == NULL || atoi(e) != 0;
    }
    const int on_device = plasma_is_device_pointer(pA);
    upload_t up = {pA, lda, on_device, !on_device && plasma_is_pageable(pA)};
    const int pipelined = pipeline_env && uplo == PlasmaLower && plasma->lookahead != 0 &&
                          !on_device;
    /* a lower-stored device matrix goes to both tile copies in one pass
     * inside the solve */
    const int direct = uplo == PlasmaLower && on_device;
    if (!pipelined && !direct)
        plasma_omp_Xlapack2desc(pA, lda, A, uplo, &sequence, &request);
    plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    if (sequence.status == PlasmaSuccess) {
        Xdsposv(plasma, uplo, A, B, X, As, Xs, R, Rnorm, Xnorm, iter,
                &sequence, &request, info, pipelined || direct ? &up : NULL);
    }
    plasma_sequence_wait(&sequence);
    plasma_omp_Xdesc2lapack(X, pX, ldx, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);

    plasma_desc_destroy(&B);
    plasma_desc_destroy(&X); plasma_desc_destroy(&R);
    plasma_desc_destroy(&Xs);
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
