/*
 * async.c -- sequence / request error model.
 *
 * plasma_request_fail / plasma_request_init / plasma_sequence_init behave as
 * the reference's control/async.c:17-40.  plasma_sequence_wait() is the GPU
 * build's synchronisation point: it waits for the context stream and folds
 * the device status word (written by the first kernel that failed) into the
 * sequence of the plasma_omp_* call that owned that kernel.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <string.h>

int plasma_request_fail(plasma_sequence_t *sequence,
                        plasma_request_t *request, int status)
{
    if (sequence) {
        sequence->request = request;
        sequence->status = status;
    }
    if (request)
        request->status = status;
    return status;
}

int plasma_request_init(plasma_request_t *request)
{
    request->status = PlasmaSuccess;
    return PlasmaSuccess;
}

int plasma_sequence_init(plasma_sequence_t *sequence)
{
    sequence->status = PlasmaSuccess;
    sequence->request = NULL;
    return PlasmaSuccess;
}

int plasma_sequence_wait(plasma_sequence_t *sequence)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    if (plasma->device < 0)
        return sequence ? sequence->status : PlasmaErrorEnvironment;

    cudaError_t err = cudaStreamSynchronize(plasma->stream);
    for (int i = 0; i < PLASMA_NUM_STREAMS; i++)
        cudaStreamSynchronize(plasma->aux[i]);
    if (err != cudaSuccess) {
        plasma_error(cudaGetErrorString(err));
        if (sequence && sequence->status == PlasmaSuccess)
            plasma_request_fail(sequence, sequence->request,
                                PlasmaErrorInternal);
        return PlasmaErrorInternal;
    }
    int cerr = plasma_take_cuda_error();
    if (cerr != 0) {
        /* a launch that never ran: its request is not known, so the error
         * goes to the sequence waited on */
        plasma_error(cudaGetErrorString((cudaError_t)cerr));
        if (sequence && sequence->status == PlasmaSuccess)
            plasma_request_fail(sequence, sequence->request, PlasmaErrorInternal);
    }
    cudaMemcpy(plasma->hstat, plasma->dstat, sizeof(plasma_devstat_t),
               cudaMemcpyDeviceToHost);
    int status = plasma->hstat->status;
    if (status != 0) {
        int call = plasma->hstat->call;
        plasma_sequence_t *owner = NULL;
        plasma_request_t *req = NULL;
        if (call > 0 && call < PLASMA_MAX_PENDING_CALLS) {
            owner = plasma->pending_seq[call];
            req = plasma->pending[call];
        }
        if (owner == NULL)
            owner = sequence;
        if (owner && owner->status == PlasmaSuccess)
            plasma_request_fail(owner, req, status);
        /* the status word is consumed: later sequences start clean */
        cudaMemset(plasma->dstat, 0, sizeof(plasma_devstat_t));
        cudaDeviceSynchronize();
    }
    memset(plasma->pending, 0, sizeof(plasma->pending));
    memset(plasma->pending_seq, 0, sizeof(plasma->pending_seq));
    plasma->next_call = 1;
    return sequence ? sequence->status : status;
}
