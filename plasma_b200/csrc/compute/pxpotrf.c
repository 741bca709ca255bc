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

void plasma_pXpotrf(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_sequence_t *sequence,
                    plasma_request_t *request, int call)
{
    (void)request;
    if (sequence->status != PlasmaSuccess)
        return;
    const int mt = A.mt;
    if (mt == 0)
        return;
    plasma_devstat_t *st = plasma->dstat;
    cudaStream_t S = plasma->stream;
    const int sms = plasma->num_sms;

    if (plasma->lookahead == 0 || mt < 3) {
        for (int k = 0; k < mt; k++) {
            plasma_cuda_potrf_tile(S, st, call, uplo, A, k, A.nb * k, NULL);
            plasma_cuda_trsm_panel(S, st, uplo, A, k, k + 1, mt, NULL);
            plasma_cuda_update(S, st, uplo, A, k, k + 1, mt, sms);
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
        cudaEventRecord(ev_panel, crit);

        /* critical: the next panel column, after the bulk stream is done
         * with it (its step k-1 update of column k+1) */
        if (have_next)
            cudaStreamWaitEvent(crit, ev_next, 0);
        plasma_cuda_update(crit, st, uplo, A, k, k + 1, k + 2, sms);

        /* bulk: the rest of step k */
        have_next = 0;
        if (k + 2 < mt) {
            cudaStreamWaitEvent(bulk, ev_panel, 0);
            plasma_cuda_update(bulk, st, uplo, A, k, k + 2, k + 3, sms);
            cudaEventRecord(ev_next, bulk);
            have_next = 1;
            if (k + 3 < mt)
                plasma_cuda_update(bulk, st, uplo, A, k, k + 3, mt, sms);
        }
    }
    cudaEventRecord(ev_crit_end, crit);
    cudaEventRecord(ev_bulk_end, bulk);
    cudaStreamWaitEvent(S, ev_crit_end, 0);
    cudaStreamWaitEvent(S, ev_bulk_end, 0);
}
