/*
 * plasma_async.h -- sequence / request error model of the asynchronous tile
 * interface.
 *
 * The two structs keep the reference's layout (include/plasma_async.h:20-27),
 * so code that allocates them on its stack keeps working.  In the GPU build a
 * plasma_omp_* call enqueues kernels on the context's CUDA stream and returns;
 * numerical failures found on the device (a non-positive pivot, an FP32
 * overflow in a precision conversion) are held in a device-side status word
 * and folded into sequence->status by plasma_sequence_wait() -- the analogue
 * of the end of the reference's "omp parallel" region.
 */
#ifndef PLASMA_ASYNC_H
#define PLASMA_ASYNC_H

#include "plasma_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    plasma_enum_t status;       /* error code of this call                 */
} plasma_request_t;

typedef struct {
    plasma_enum_t status;       /* first error of the sequence             */
    plasma_request_t *request;  /* the request that failed                 */
} plasma_sequence_t;

/* reference control/async.c:17-25 */
int plasma_request_fail(plasma_sequence_t *sequence,
                        plasma_request_t *request, int status);
/* reference control/async.c:28-32 */
int plasma_request_init(plasma_request_t *request);
/* reference control/async.c:35-40 */
int plasma_sequence_init(plasma_sequence_t *sequence);

/*
 * GPU-build addition: waits for every kernel enqueued by plasma_omp_* calls
 * on the context stream and copies the device status into
 * sequence->status (only if the sequence has not failed already).  Returns
 * the resulting sequence->status.  The reference synchronises implicitly at
 * the end of its parallel region (compute/zpotrf.c:130-141).
 */
int plasma_sequence_wait(plasma_sequence_t *sequence);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_ASYNC_H */
