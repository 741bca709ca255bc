/*
 * pxpotrf.c -- the tile Cholesky DAG on CUDA streams.
 *
 * Same loop nest as the reference's plasma_pzpotrf (compute/pzpotrf.c:37-80
 * for lower storage, :84-126 for upper): for each step k, POTRF of tile
 * (k,k), TRSM of the tiles below it, then SYRK/GEMM on the trailing matrix.
 * The reference hands every tile operation to OpenMP as a task and lets the
 * depend() clauses order them.  Here one kernel covers a whole tile step and
 * the edges of the DAG become stream order plus events:
 *
 *   crit stream (high priority):  POTRF(k) -> TRSM(k) -> [wait N(k-1)]
 *                                 UPDATE(k, column k+1)
 *   bulk stream (low priority):   [wait P(k)] UPDATE(k, column k+2) -> N(k)
 *                                 UPDATE(k, columns k+3 ..)
 *
 * so the panel of step k+1 is factored while the bulk of step k's update is
 * still running (look-ahead of depth 1).  Column k+2 is split off the bulk
 * update so that the critical stream only waits for the part it touches.
 * With PlasmaLookahead = 0 everything runs in program order on one stream.
 *
 * Failure handling: POTRF(k) writes the device status word with
 * info = A.nb*k + j (compute/pzpotrf.c:44); every later kernel reads the word
 * first and returns, like the reference's tasks test sequence->status.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <stdint.h>

typedef struct {
    plasma_devstat_t *st;
    plasma_enum_t uplo;
    plasma_desc_t A;
    int sms;
    int mode;          /* PLASMA_TC_* product precision of the tensor-core
                          update, or 0 for the DMMA/SIMT update            */
    char *panel[2];    /* rounded copies of panels k (alternating buffers)   */
} walk_t;

static void update(walk_t *w, cudaStream_t s, int k, int nlo, int nhi)
{
    if (w->mode) {
        if (plasma_cuda_update_tc(s, w->st, w->mode, w->A, k, nlo, nhi,
                                  w->panel[k & 1], w->sms))
            return;
    }
    plasma_cuda_update(s, w->st, w->uplo, w->A, k, nlo, nhi, w->sms);
}

void plasma_pXpotrf(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_sequence_t *sequence,
                    plasma_request_t *request, int call)
{
    plasma_pXpotrf_mode(plasma, uplo, A, sequence, request, call, 0);
}

void plasma_pXpotrf_mode(plasma_context_t *plasma, plasma_enum_t uplo,
                         plasma_desc_t A, plasma_sequence_t *sequence,
                         plasma_request_t *request, int call, int mode)
{
    if (sequence->status != PlasmaSuccess)
        return;
    const int mt = A.mt;
    if (mt == 0)
        return;
    plasma_devstat_t *st = plasma->dstat;
    cudaStream_t S = plasma->stream;

    walk_t w;
    w.st = st;
    w.uplo = uplo;
    w.A = A;
    w.sms = plasma->num_sms;
    w.mode = 0;
    w.panel[0] = w.panel[1] = NULL;
    /* FP32 factors: every mode runs its update on the tensor cores when the
     * tiles allow it (FP32 as the three-product TF32 split) */
    int tc = mode == PlasmaFactorTF32 ? PLASMA_TC_TF32
           : mode == PlasmaFactorBF16 ? PLASMA_TC_BF16 : PLASMA_TC_TF32X3;
    if (plasma_cuda_update_tc_ok(A, uplo)) {
        size_t one = (plasma_cuda_panel_bytes(tc, A) + 1023) & ~(size_t)1023;
        char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_MIXED, 2 * one + 1024);
        if (buf != NULL) {
            buf = (char *)(((uintptr_t)buf + 1023) & ~(uintptr_t)1023);
            w.mode = tc;
            w.panel[0] = buf;
            w.panel[1] = buf + one;
        }
    }
    /* FP32 panels: TF32 products next to a TF32/BF16 update, else the
     * FP32-accurate split */
    if (A.precision == PlasmaRealFloat)
        plasma_cuda_panel_set_split(w.mode == PLASMA_TC_TF32 ||
                                    w.mode == PLASMA_TC_BF16 ? 1 : 3);

    if (plasma->lookahead == 0 || mt < 3) {
        for (int k = 0; k < mt; k++) {
            plasma_cuda_potrf_tile(S, st, call, uplo, A, k, A.nb * k, NULL);
            plasma_cuda_trsm_panel(S, st, uplo, A, k, k + 1, mt, NULL);
            if (w.mode)
                plasma_cuda_panel_round(S, st, w.mode, A, k, w.panel[k & 1]);
            update(&w, S, k, k + 1, mt);
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

    int have_next = 0;   /* N(k-1) was recorded */
    for (int k = 0; k < mt; k++) {
        plasma_cuda_potrf_tile(crit, st, call, uplo, A, k, A.nb * k, NULL);
        plasma_cuda_trsm_panel(crit, st, uplo, A, k, k + 1, mt, NULL);
        if (k + 1 >= mt)
            break;
        /* the bulk stream is done with column k+1 (its step k-1 update) and,
         * since N(k-1) follows the whole step k-2 update on that stream, with
         * the panel buffer that the rounded copy of panel k is about to reuse */
        if (have_next)
            cudaStreamWaitEvent(crit, ev_next, 0);
        if (w.mode)
            plasma_cuda_panel_round(crit, st, w.mode, A, k, w.panel[k & 1]);
        cudaEventRecord(ev_panel, crit);

        /* critical: the next panel column */
        update(&w, crit, k, k + 1, k + 2);

        /* bulk: the rest of step k */
        have_next = 0;
        if (k + 2 < mt) {
            cudaStreamWaitEvent(bulk, ev_panel, 0);
            update(&w, bulk, k, k + 2, k + 3);
            cudaEventRecord(ev_next, bulk);
            have_next = 1;
            if (k + 3 < mt)
                update(&w, bulk, k, k + 3, mt);
        }
    }
    cudaEventRecord(ev_crit_end, crit);
    cudaEventRecord(ev_bulk_end, bulk);
    cudaStreamWaitEvent(S, ev_crit_end, 0);
    cudaStreamWaitEvent(S, ev_bulk_end, 0);
}
