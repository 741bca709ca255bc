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
 * A matrix whose tile columns are still arriving (plasma_pXpotrf_arrivals)
 * replaces the bulk stream by one stream per group of columns (walk_groups).
 *
 * Failure handling: POTRF(k) writes the device status word with
 * info = A.nb*k + j (compute/pzpotrf.c:44); every later kernel reads the word
 * first and returns, like the reference's tasks test sequence->status.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    plasma_devstat_t *st;
    plasma_enum_t uplo;
    plasma_desc_t A;
    int sms;
    int mode;          /* PLASMA_TC_* product precision of the tensor-core
                          update, or 0 for the DMMA/SIMT update            */
    int full;          /* panel copies: every panel (1) or two buffers (0) */
    char *panel[3];    /* rounded copies of panel k (buffer k % 3, or all) */
    char *wimg;        /* operand image of the diagonal tile for the
                          tensor-core panel solve (plasma_cuda_trsm_tc)    */
} walk_t;

/* FP32 factors: every mode runs its update on the tensor cores when the
 * tiles allow it.  FP32 accuracy comes from a split of the panel: three
 * TF32 products of a two-part split, or with PLASMA_FP32_SPLIT=bf16x6
 * (256-wide tiles) six BF16 products of a three-part split, which moves
 * 6 instead of 8 operand bytes per element at the same tensor time. */
static int tc_mode(plasma_desc_t A, int mode)
{
    static int split_env = -1;
    if (split_env < 0) {
        const char *e = getenv("PLASMA_FP32_SPLIT");
        split_env = (e != NULL && strcmp(e, "bf16x6") == 0) ? 1 : 0;
    }
    return mode == PlasmaFactorTF32 ? PLASMA_TC_TF32
         : mode == PlasmaFactorBF16 ? PLASMA_TC_BF16
         : (A.mb == 256 && split_env) ? PLASMA_TC_BF16X6 : PLASMA_TC_TF32X3;
}

/* the panel copies: three buffers, or one holding every panel; then the
 * operand image of the panel solve.  Panel k's copy is written by the
 * solve of step k (or by plasma_cuda_panel_round right after it); with
 * three buffers the one it reuses was last read by the step k-3 update,
 * which the critical stream has waited for (N(k-2)) before step k. */
static size_t panel_scratch_bytes(plasma_desc_t A, int tc, int full)
{
    const size_t one = (plasma_cuda_panel_bytes(tc, A, full) + 1023) & ~(size_t)1023;
    const size_t wimg = (plasma_cuda_trsm_tc_bytes(A.nb) + 1023) & ~(size_t)1023;
    return (full ? 1 : 3) * one + wimg + 1024;
}

void plasma_pXpotrf_reserve(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                            int mode, int full)
{
    if (plasma_cuda_update_tc_ok(A, uplo))
        plasma_scratch(plasma, PLASMA_SLOT_MIXED, panel_scratch_bytes(A, tc_mode(A, mode), full));
}

static void *panel_buf(walk_t *w, int k)
{
    return w->full ? w->panel[0] : w->panel[k % 3];
}

static void update(walk_t *w, cudaStream_t s, int k, int nlo, int nhi)
{
    if (w->mode) {
        if (plasma_cuda_update_tc(s, w->st, w->mode, w->A, k, nlo, nhi,
                                  panel_buf(w, k), w->full, w->sms))
            return;
    }
    plasma_cuda_update(s, w->st, w->uplo, w->A, k, nlo, nhi, w->sms);
}

static void round_panel(walk_t *w, cudaStream_t s, int k)
{
    if (w->mode)
        plasma_cuda_panel_round(s, w->st, w->mode, w->A, k, panel_buf(w, k), w->full);
}

/* The panel solve of step k: on the tensor cores next to a tensor-core
 * update (which then also writes the rounded panel copies when the update
 * takes TF32 operands), else the generic kernels.  Returns 1 when the
 * panel copies are written. */
static int trsm(walk_t *w, cudaStream_t s, int k)
{
    if (w->mode && w->wimg != NULL) {
        const int r = plasma_cuda_trsm_tc(s, w->st, w->mode, w->A, k, k + 1, w->A.mt,
                                          w->wimg, panel_buf(w, k), w->full);
        if (r)
            return r == 2;
    }
    plasma_cuda_trsm_panel(s, w->st, w->uplo, w->A, k, k + 1, w->A.mt, NULL);
    return 0;
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
    plasma_pXpotrf_arrivals(plasma, uplo, A, sequence, request, call, mode, 0, NULL, NULL);
}

/* The arriving-columns DAG: one update stream per column group.  At step k
 * the stream of group g applies panel k to its columns from k+2 on, after
 * the group has arrived; a group that arrives late works through the steps
 * it missed from the kept panel copies while the critical stream goes on
 * with the columns that are in.  The stream holding column k+2 splits it
 * off and records N(k), which the critical stream waits for at step k+1,
 * as in the one-bulk-stream DAG.
 *
 * Groups outnumber the streams: group g runs on stream g mod S.  It starts
 * (waits for its arrival, then applies panels 0 .. k-1 in one stretch) at
 * the step k where group g-S has taken its last update, step
 * gstart[g-S+1] - 3; that is always before group g's first column needs
 * its first update (step gstart[g] - 2), since every group holds a column. */
static void walk_groups(plasma_context_t *plasma, walk_t *w, int call, int ngroups,
                        const int *gstart, const cudaEvent_t *arrive)
{
    plasma_devstat_t *st = w->st;
    plasma_enum_t uplo = w->uplo;
    plasma_desc_t A = w->A;
    const int mt = A.mt;
    const int nstreams = ngroups < PLASMA_GROUP_STREAMS ? ngroups : PLASMA_GROUP_STREAMS;
    cudaStream_t S = plasma->stream;
    cudaStream_t crit = plasma->aux[0];
    cudaEvent_t ev_start = plasma->ev[0];
    cudaEvent_t ev_panel = plasma->ev[1];
    cudaEvent_t ev_next = plasma->ev[2];
    cudaEvent_t ev_end = plasma->ev[3];

    cudaEventRecord(ev_start, S);
    cudaStreamWaitEvent(crit, ev_start, 0);
    for (int s = 0; s < nstreams; s++) {
        cudaStream_t gs = plasma->aux[3 + s];
        cudaStreamWaitEvent(gs, ev_start, 0);
        cudaStreamWaitEvent(gs, arrive[s], 0);   /* groups 0 .. nstreams-1 */
    }
    cudaStreamWaitEvent(crit, arrive[0], 0);

    int active = nstreams;           /* groups [0, active) have started */
    int have_next = 0;
    int gk = 0;                      /* group of column k + 1 */
    for (int k = 0; k < mt; k++) {
        plasma_cuda_potrf_tile(crit, st, call, uplo, A, k, A.nb * k, NULL);
        const int rounded = trsm(w, crit, k);
        if (k + 1 >= mt)
            break;
        while (gstart[gk + 1] <= k + 1) gk++;
        cudaStreamWaitEvent(crit, arrive[gk], 0);
        if (have_next)
            cudaStreamWaitEvent(crit, ev_next, 0);
        if (!rounded)
            round_panel(w, crit, k);
        cudaEventRecord(ev_panel, crit);
        update(w, crit, k, k + 1, k + 2);

        /* groups whose stream came free: arrival, then the missed steps
         * (panels 0 .. k-1 are done once panel k is) */
        while (active < ngroups && gstart[active - nstreams + 1] - 3 < k) {
            const int g = active++;
            cudaStream_t gs = plasma->aux[3 + g % nstreams];
            cudaStreamWaitEvent(gs, arrive[g], 0);
            cudaStreamWaitEvent(gs, ev_panel, 0);
            for (int kk = 0; kk < k; kk++)
                update(w, gs, kk, gstart[g], gstart[g + 1]);
        }

        have_next = 0;
        for (int g = gk; g < active; g++) {
            const int hi = gstart[g + 1];
            const int lo = gstart[g] > k + 2 ? gstart[g] : k + 2;
            if (lo >= hi)
                continue;
            cudaStream_t gs = plasma->aux[3 + g % nstreams];
            cudaStreamWaitEvent(gs, ev_panel, 0);
            if (lo == k + 2) {
                update(w, gs, k, k + 2, k + 3);
                cudaEventRecord(ev_next, gs);
                have_next = 1;
                if (k + 3 < hi)
                    update(w, gs, k, k + 3, hi);
            } else {
                update(w, gs, k, lo, hi);
            }
        }
    }
    cudaEventRecord(ev_end, crit);
    cudaStreamWaitEvent(S, ev_end, 0);
    for (int s = 0; s < nstreams; s++) {
        cudaEventRecord(ev_end, plasma->aux[3 + s]);
        cudaStreamWaitEvent(S, ev_end, 0);
    }
}

void plasma_pXpotrf_arrivals(plasma_context_t *plasma, plasma_enum_t uplo,
                             plasma_desc_t A, plasma_sequence_t *sequence,
                             plasma_request_t *request, int call, int mode,
                             int ngroups, const int *gstart, const cudaEvent_t *arrive)
{
    if (sequence->status != PlasmaSuccess)
        return;
    const int mt = A.mt;
    if (mt == 0)
        return;
    plasma_devstat_t *st = plasma->dstat;
    cudaStream_t S = plasma->stream;
    if (ngroups > PLASMA_MAX_GROUPS) {
        /* more groups than arrival slots: wait for all of them */
        for (int g = 0; g < ngroups; g++)
            cudaStreamWaitEvent(S, arrive[g], 0);
        ngroups = 0;
    }
    const int grouped = ngroups > 0 && plasma->lookahead != 0 && mt >= 3;
    if (ngroups > 0 && !grouped)
        for (int g = 0; g < ngroups; g++)
            cudaStreamWaitEvent(S, arrive[g], 0);

    walk_t w;
    w.st = st;
    w.uplo = uplo;
    w.A = A;
    w.sms = plasma->num_sms;
    w.mode = 0;
    w.full = grouped;
    w.panel[0] = w.panel[1] = w.panel[2] = NULL;
    w.wimg = NULL;
    int tc = tc_mode(A, mode);
    if (plasma_cuda_update_tc_ok(A, uplo)) {
        char *buf = (char *)plasma_scratch(plasma, PLASMA_SLOT_MIXED,
                                           panel_scratch_bytes(A, tc, w.full));
        if (buf != NULL) {
            const size_t one = (plasma_cuda_panel_bytes(tc, A, w.full) + 1023) & ~(size_t)1023;
            buf = (char *)(((uintptr_t)buf + 1023) & ~(uintptr_t)1023);
            w.mode = tc;
            w.panel[0] = buf;
            w.panel[1] = buf + one;
            w.panel[2] = buf + 2 * one;
            w.wimg = buf + (w.full ? 1 : 3) * one;
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
            if (!trsm(&w, S, k))
                round_panel(&w, S, k);
            update(&w, S, k, k + 1, mt);
        }
        return;
    }

    if (grouped) {
        walk_groups(plasma, &w, call, ngroups, gstart, arrive);
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
        const int rounded = trsm(&w, crit, k);
        if (k + 1 >= mt)
            break;
        /* the bulk stream is done with column k+1 (its step k-1 update) */
        if (have_next)
            cudaStreamWaitEvent(crit, ev_next, 0);
        if (!rounded)
            round_panel(&w, crit, k);
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
