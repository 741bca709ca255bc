/*
 * pbtrf.c -- Cholesky factorization and solve of an SPD band matrix:
 * plasma_{d,s}pbtrf (compute/zpbtrf.c:77-158, :202-242), plasma_{d,s}pbtrs
 * (compute/zpbtrs.c:81-182, :236-295), plasma_{d,s}pbsv (compute/zpbsv.c:
 * 92-193, :242-302), their plasma_omp_* forms, and the band layout
 * converters plasma_omp_{d,s}{pb2desc,desc2pb} (compute/zpb2desc.c,
 * zdesc2pb.c).
 *
 * Interface and semantics as in the reference: LAPACK band storage
 * AB(kd+1+i-j, j) = A(i,j) (upper) or AB(1+i-j, j) = A(i,j) (lower), the
 * reference's argument codes (including its numbering for pbtrs: kd -4,
 * nrhs -5, ldab -7, ldb -10), quick returns, a band tile descriptor with
 * lm = nb*(1 + ceil(kd/nb)) rows and kl = ku = kd (so a band wider than the
 * matrix, kd >= n, fails the descriptor check with PlasmaErrorIllegalValue as
 * in the reference), and info = i > 0 when the leading minor of order i is
 * not positive.  After a failure AB is left as it was.
 *
 * The factorization is the reference's band tile loop (compute/pzpbtrf.c:
 * 37-80 lower, :84-118 upper) -- POTRF of tile (k,k), TRSM of the kt-1 tiles
 * below it, SYRK/GEMM on the kt-1 x kt-1 trailing window -- run on the same
 * tile-step kernels as the dense factorization: each step passes them a view
 * of the band descriptor whose last tile row is k+kt-1, so the dense
 * kernels' row range (the view's mt) is the band's.  The steps follow the
 * dense look-ahead DAG on two streams (compute/pxpotrf.c): the critical
 * stream factors panel k+1 while the bulk stream finishes step k's window.
 * The solves are the tile sweeps of potrs restricted to the band's tiles
 * (cuda/solve.cu), the reference's pztbsm.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>

/* tiles of a band tile column from the diagonal outwards (logical lower
 * view: below the diagonal for lower storage, right of it for upper) */
static int band_tiles(plasma_enum_t uplo, plasma_desc_t A)
{
    return uplo == PlasmaLower ? A.klt : A.kut;
}

/* The band with its tile rows and columns cut at r: the tile kernels take
 * their row range from the view's mt. */
static plasma_desc_t band_rows(plasma_desc_t A, int r)
{
    plasma_desc_t V = A;
    V.m = imin(A.m, r * A.mb);
    V.n = imin(A.n, r * A.nb);
    V.mt = (V.m + A.mb - 1) / A.mb;
    V.nt = (V.n + A.nb - 1) / A.nb;
    return V;
}

static void band_update(plasma_context_t *plasma, cudaStream_t s, plasma_enum_t uplo,
                        plasma_desc_t V, int k, int nlo, int nhi)
{
    if (nhi > nlo)
        plasma_cuda_update(s, plasma->dstat, uplo, V, k, nlo, nhi, plasma->num_sms);
}

void plasma_pXpbtrf(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                    plasma_sequence_t *sequence, plasma_request_t *request, int call)
{
    (void)request;
    if (sequence->status != PlasmaSuccess)
        return;
    const int mt = A.mt;
    if (mt == 0)
        return;
    const int kt = band_tiles(uplo, A);
    plasma_devstat_t *st = plasma->dstat;
    cudaStream_t S = plasma->stream;
    /* FP32 band factors are FP32-accurate: the split panel kernels */
    if (A.precision == PlasmaRealFloat)
        plasma_cuda_panel_set_split(3);

    if (plasma->lookahead == 0 || mt < 3) {
        for (int k = 0; k < mt; k++) {
            const int r = imin(mt, k + kt);
            plasma_desc_t V = band_rows(A, r);
            plasma_cuda_potrf_tile(S, st, call, uplo, V, k, A.nb * k, NULL);
            plasma_cuda_trsm_panel(S, st, uplo, V, k, k + 1, r, NULL);
            band_update(plasma, S, uplo, V, k, k + 1, r);
        }
        return;
    }

    cudaStream_t crit = plasma->aux[0];
    cudaStream_t bulk = plasma->aux[1];
    cudaEvent_t ev_start = plasma->ev[0];
    cudaEvent_t ev_panel = plasma->ev[1];     /* P(k): panel k solved     */
    cudaEvent_t ev_next = plasma->ev[2];      /* N(k): column k+2 updated */
    cudaEvent_t ev_crit_end = plasma->ev[3];
    cudaEvent_t ev_bulk_end = plasma->ev[4];

    cudaEventRecord(ev_start, S);
    cudaStreamWaitEvent(crit, ev_start, 0);
    cudaStreamWaitEvent(bulk, ev_start, 0);

    /* Step k touches tile columns [k+1, r) and rows below them up to r-1.
     * Column k+1 is updated on the critical stream; column k+2 first on
     * the bulk stream, which records N(k) before the rest of the window;
     * the critical stream waits for N(k-1) before it updates column k+1 at
     * step k (the dense DAG's edges, cut to the band). */
    int have_next = 0;
    for (int k = 0; k < mt; k++) {
        const int r = imin(mt, k + kt);
        plasma_desc_t V = band_rows(A, r);
        plasma_cuda_potrf_tile(crit, st, call, uplo, V, k, A.nb * k, NULL);
        plasma_cuda_trsm_panel(crit, st, uplo, V, k, k + 1, r, NULL);
        if (k + 1 >= mt)
            break;
        if (have_next)
            cudaStreamWaitEvent(crit, ev_next, 0);
        cudaEventRecord(ev_panel, crit);
        band_update(plasma, crit, uplo, V, k, k + 1, imin(k + 2, r));
        have_next = 0;
        if (k + 2 < r) {
            cudaStreamWaitEvent(bulk, ev_panel, 0);
            band_update(plasma, bulk, uplo, V, k, k + 2, k + 3);
            cudaEventRecord(ev_next, bulk);
            have_next = 1;
            band_update(plasma, bulk, uplo, V, k, k + 3, r);
        }
    }
    cudaEventRecord(ev_crit_end, crit);
    cudaEventRecord(ev_bulk_end, bulk);
    cudaStreamWaitEvent(S, ev_crit_end, 0);
    cudaStreamWaitEvent(S, ev_bulk_end, 0);
}

/* the two band sweeps (compute/zpbtrs.c:280-294) */
void plasma_pXpbtrs(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                    plasma_desc_t B, plasma_sequence_t *sequence, plasma_request_t *request)
{
    if (sequence->status != PlasmaSuccess)
        return;
    size_t elem = plasma_element_size(A.precision);
    void *W = plasma_scratch(plasma, PLASMA_SLOT_WORK, (size_t)A.mt * A.mb * A.mb * elem);
    if (W == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_cuda_trsm_sweep(plasma->stream, plasma->dstat, uplo, PlasmaNoTrans, A, B, W, 0);
    plasma_cuda_trsm_sweep(plasma->stream, plasma->dstat, uplo, PlasmaTrans, A, B, W, 1);
}

/* ------------------------------------------------------------------ checks */

static int check_band(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t AB,
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
    /* the band storage must hold the uplo triangle's tiles */
    if (plasma_desc_check(AB) != PlasmaSuccess || AB.type != PlasmaGeneralBand ||
        (AB.uplo != uplo && AB.uplo != PlasmaGeneral)) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    return 1;
}

static int check_gpu(plasma_context_t *plasma, plasma_desc_t AB,
                     plasma_sequence_t *sequence, plasma_request_t *request)
{
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    if (AB.mb != AB.nb || AB.mb > (AB.precision == PlasmaRealDouble ? 512 : 1024)) {
        plasma_error("tile size not supported by the GPU kernels");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return 0;
    }
    return 1;
}

/* --------------------------------------------------------- async interface */

static void plasma_omp_Xpbtrf(plasma_enum_t uplo, plasma_desc_t AB,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_band(plasma, uplo, AB, sequence, request))
        return;
    if (AB.m == 0)
        return;
    if (!check_gpu(plasma, AB, sequence, request))
        return;
    int call = plasma_call_begin(plasma, sequence, request);
    plasma_pXpbtrf(plasma, uplo, AB, sequence, request, call);
}

static void plasma_omp_Xpbtrs(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                              plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_band(plasma, uplo, AB, sequence, request))
        return;
    if (plasma_desc_check(B) != PlasmaSuccess) {
        plasma_error("invalid B");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (AB.n == 0 || B.n == 0)
        return;
    if (!check_gpu(plasma, AB, sequence, request))
        return;
    plasma_call_begin(plasma, sequence, request);
    plasma_pXpbtrs(plasma, uplo, AB, B, sequence, request);
}

static void plasma_omp_Xpbsv(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                             plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_band(plasma, uplo, AB, sequence, request))
        return;
    if (plasma_desc_check(B) != PlasmaSuccess) {
        plasma_error("invalid B");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (AB.n == 0 || B.n == 0)
        return;
    if (!check_gpu(plasma, AB, sequence, request))
        return;
    int call = plasma_call_begin(plasma, sequence, request);
    plasma_pXpbtrf(plasma, uplo, AB, sequence, request, call);
    plasma_pXpbtrs(plasma, uplo, AB, B, sequence, request);
}

/* ------------------------------------------------------- layout converters */

/* rows of LAPACK band storage that hold the band (kd+1) */
static int band_height(plasma_desc_t A)
{
    return (A.uplo == PlasmaLower ? A.kl : A.ku) + 1;
}

static int check_pb(plasma_context_t *plasma, const void *pAB, int ldab, plasma_desc_t A,
                    plasma_sequence_t *sequence, plasma_request_t *request)
{
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return 0;
    }
    if (pAB == NULL) {
        plasma_error("NULL A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma_desc_check(A) != PlasmaSuccess || A.type != PlasmaGeneralBand) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return 0;
    }
    if (A.uplo != PlasmaLower && A.uplo != PlasmaUpper) {
        /* general band storage (kl extra rows for LU fill) is not handled */
        plasma_error("band storage must be upper or lower");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return 0;
    }
    if (ldab < band_height(A)) {
        plasma_error("illegal value of ldab");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    return sequence->status == PlasmaSuccess && A.m > 0 && A.n > 0;
}

void plasma_omp_Xpb2desc(const void *pAB, int ldab, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_pb(plasma, pAB, ldab, A, sequence, request))
        return;
    const void *src = pAB;
    int ld = ldab;
    if (!plasma_is_device_pointer(pAB)) {
        /* stage the kd+1 band rows of every column */
        size_t elem = plasma_element_size(A.precision);
        ld = band_height(A);
        void *buf = plasma_scratch(plasma, PLASMA_SLOT_STAGING, (size_t)ld * A.n * elem);
        if (buf == NULL) {
            plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
            return;
        }
        plasma_copy_2d(plasma, plasma->stream, buf, (size_t)ld * elem, pAB,
                       (size_t)ldab * elem, (size_t)ld * elem, (size_t)A.n,
                       cudaMemcpyHostToDevice, plasma_is_pageable(pAB));
        src = buf;
    }
    plasma_cuda_band_to_tile(plasma->stream, plasma->dstat, A, src, ld);
}

void plasma_omp_Xdesc2pb(plasma_desc_t A, void *pAB, int ldab,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_pb(plasma, pAB, ldab, A, sequence, request))
        return;
    if (plasma_is_device_pointer(pAB)) {
        plasma_cuda_tile_to_band(plasma->stream, plasma->dstat, A, pAB, ldab);
        return;
    }
    size_t elem = plasma_element_size(A.precision);
    const int ld = band_height(A);
    char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_STAGING, (size_t)ld * A.n * elem);
    if (buf == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    /* The kd columns at the corner of the band (the last ones for lower
     * storage, the first ones for upper) hold positions outside the matrix
     * that LAPACK leaves alone: they travel up first so that the copy back
     * returns them unchanged. */
    const int nc = imin(A.n, ld - 1);
    const int c0 = A.uplo == PlasmaLower ? A.n - nc : 0;
    const int pageable = plasma_is_pageable(pAB);
    if (nc > 0)
        plasma_copy_2d(plasma, plasma->stream, buf + (size_t)c0 * ld * elem, (size_t)ld * elem,
                       (const char *)pAB + (size_t)c0 * ldab * elem, (size_t)ldab * elem,
                       (size_t)ld * elem, (size_t)nc, cudaMemcpyHostToDevice, pageable);
    plasma_cuda_tile_to_band(plasma->stream, plasma->dstat, A, buf, ld);
    plasma_copy_2d(plasma, plasma->stream, pAB, (size_t)ldab * elem, buf, (size_t)ld * elem,
                   (size_t)ld * elem, (size_t)A.n, cudaMemcpyDeviceToHost, pageable);
    cudaStreamSynchronize(plasma->stream);
}

/* ------------------------------------------------------ LAPACK interface */

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request);
/* The band tile copy of AB in the context's kept slot (the reference
 * allocates it per call with plasma_desc_general_band_create). */
static int band_desc(plasma_context_t *plasma, plasma_enum_t prec, plasma_enum_t uplo,
                     int n, int kd, plasma_desc_t *AB)
{
    const int nb = plasma->nb;
    const int lm = nb * (1 + (kd + nb - 1) / nb);
    int rc = plasma_desc_general_band_init(prec, uplo, NULL, nb, nb, lm, n, 0, 0, n, n,
                                           kd, kd, AB);
    if (rc != PlasmaSuccess)
        return rc;
    if (plasma_desc_check(*AB) != PlasmaSuccess) {
        plasma_error("plasma_desc_general_band_create() failed");
        return PlasmaErrorIllegalValue;
    }
    AB->matrix = plasma_scratch(plasma, PLASMA_SLOT_DESC_A, plasma_desc_storage_bytes(*AB));
    return AB->matrix == NULL ? PlasmaErrorOutOfMemory : PlasmaSuccess;
}

enum { OP_TRF, OP_TRS, OP_SV };

static int Xband(plasma_enum_t prec, int op, plasma_enum_t uplo, int n, int kd, int nrhs,
                 void *pAB, int ldab, void *pB, int ldb)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    /* the reference's argument codes per routine */
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        return -1;
    }
    if (n < 0) {
        plasma_error("illegal value of n");
        return -2;
    }
    if (kd < 0) {
        plasma_error("illegal value of kd");
        return op == OP_TRS ? -4 : -3;
    }
    if (op != OP_TRF && nrhs < 0) {
        plasma_error("illegal value of nrhs");
        return op == OP_TRS ? -5 : -4;
    }
    if (ldab < imax(1, kd + 1)) {
        plasma_error("illegal value of ldab");
        return op == OP_TRF ? -5 : op == OP_TRS ? -7 : -6;
    }
    if (op != OP_TRF && ldb < imax(1, n)) {
        plasma_error("illegal value of ldb");
        return op == OP_TRS ? -10 : -8;
    }
    if (op == OP_TRF ? n == 0 : op == OP_TRS ? imax(n, nrhs) == 0 : imin(n, nrhs) == 0)
        return PlasmaSuccess;
    if (plasma->device < 0)
        return PlasmaErrorEnvironment;
    if (plasma->tuning)
        plasma_tune_pbtrf(plasma, prec, n, kd);

    plasma_desc_t AB, B;
    int retval = band_desc(plasma, prec, uplo, n, kd, &AB);
    if (retval != PlasmaSuccess)
        return retval;
    const int nb = plasma->nb;
    if (op != OP_TRF) {
        retval = plasma_desc_general_create(prec, nb, nb, n, nrhs, 0, 0, n, nrhs, &B);
        if (retval != PlasmaSuccess)
            return retval;
    }
    plasma_sequence_t sequence;
    plasma_request_t request;
    plasma_sequence_init(&sequence);
    plasma_request_init(&request);

    plasma_omp_Xpb2desc(pAB, ldab, AB, &sequence, &request);
    if (op != OP_TRF)
        plasma_omp_Xlapack2desc(pB, ldb, B, PlasmaGeneral, &sequence, &request);
    if (op == OP_TRF)
        plasma_omp_Xpbtrf(uplo, AB, &sequence, &request);
    else if (op == OP_TRS)
        plasma_omp_Xpbtrs(uplo, AB, B, &sequence, &request);
    else
        plasma_omp_Xpbsv(uplo, AB, B, &sequence, &request);
    /* after a failure the conversions back see the failed sequence and
     * leave AB and B as they were */
    plasma_sequence_wait(&sequence);
    if (op != OP_TRS)
        plasma_omp_Xdesc2pb(AB, pAB, ldab, &sequence, &request);
    if (op != OP_TRF)
        plasma_omp_Xdesc2lapack(B, pB, ldb, PlasmaGeneral, &sequence, &request);
    plasma_sequence_wait(&sequence);
    if (op != OP_TRF)
        plasma_desc_destroy(&B);
    return sequence.status;
}

int plasma_dpbtrf(plasma_enum_t uplo, int n, int kd, double *pAB, int ldab)
{
    return Xband(PlasmaRealDouble, OP_TRF, uplo, n, kd, 0, pAB, ldab, NULL, 1);
}

int plasma_spbtrf(plasma_enum_t uplo, int n, int kd, float *pAB, int ldab)
{
    return Xband(PlasmaRealFloat, OP_TRF, uplo, n, kd, 0, pAB, ldab, NULL, 1);
}

int plasma_dpbtrs(plasma_enum_t uplo, int n, int kd, int nrhs, double *pAB, int ldab,
                  double *pB, int ldb)
{
    return Xband(PlasmaRealDouble, OP_TRS, uplo, n, kd, nrhs, pAB, ldab, pB, ldb);
}

int plasma_spbtrs(plasma_enum_t uplo, int n, int kd, int nrhs, float *pAB, int ldab,
                  float *pB, int ldb)
{
    return Xband(PlasmaRealFloat, OP_TRS, uplo, n, kd, nrhs, pAB, ldab, pB, ldb);
}

int plasma_dpbsv(plasma_enum_t uplo, int n, int kd, int nrhs, double *pAB, int ldab,
                 double *pB, int ldb)
{
    return Xband(PlasmaRealDouble, OP_SV, uplo, n, kd, nrhs, pAB, ldab, pB, ldb);
}

int plasma_spbsv(plasma_enum_t uplo, int n, int kd, int nrhs, float *pAB, int ldab,
                 float *pB, int ldb)
{
    return Xband(PlasmaRealFloat, OP_SV, uplo, n, kd, nrhs, pAB, ldab, pB, ldb);
}

void plasma_omp_dpbtrf(plasma_enum_t uplo, plasma_desc_t AB, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpbtrf(uplo, AB, sequence, request);
}

void plasma_omp_spbtrf(plasma_enum_t uplo, plasma_desc_t AB, plasma_sequence_t *sequence,
                       plasma_request_t *request)
{
    plasma_omp_Xpbtrf(uplo, AB, sequence, request);
}

void plasma_omp_dpbtrs(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpbtrs(uplo, AB, B, sequence, request);
}

void plasma_omp_spbtrs(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                       plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpbtrs(uplo, AB, B, sequence, request);
}

void plasma_omp_dpbsv(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpbsv(uplo, AB, B, sequence, request);
}

void plasma_omp_spbsv(plasma_enum_t uplo, plasma_desc_t AB, plasma_desc_t B,
                      plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpbsv(uplo, AB, B, sequence, request);
}

void plasma_omp_dpb2desc(double *pAB, int ldab, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpb2desc(pAB, ldab, A, sequence, request);
}

void plasma_omp_spb2desc(float *pAB, int ldab, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xpb2desc(pAB, ldab, A, sequence, request);
}

void plasma_omp_ddesc2pb(plasma_desc_t A, double *pAB, int ldab,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2pb(A, pAB, ldab, sequence, request);
}

void plasma_omp_sdesc2pb(plasma_desc_t A, float *pAB, int ldab,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2pb(A, pAB, ldab, sequence, request);
}
