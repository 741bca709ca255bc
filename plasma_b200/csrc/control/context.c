/*
 * context.c -- library lifetime and configuration.
 *
 * Follows the reference's control/context.c:
 *   plasma_init      :30-47   (second init -> PlasmaErrorNotInitialized)
 *   plasma_finalize  :54-71
 *   plasma_set       :78-127  (PlasmaNb <= 0 -> PlasmaErrorIllegalValue)
 *   plasma_get       :133-159
 *   defaults         :165-180 (nb 256, ib 64, tuning enabled)
 * There is one global context, as in the reference (:22-23).  In place of the
 * OpenMP team the context owns a CUDA device, a sequence stream, look-ahead
 * streams and the device status word that kernels use for cooperative
 * cancellation.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int plasma_initialized_g = 0;
static plasma_context_t plasma_context_g;
static int plasma_device_request_g = 0;   /* PlasmaDevice set before init */
long long plasma_launch_count_g = 0;
long long plasma_alloc_count_g = 0;
static int plasma_cuda_error_g = 0;        /* first unreported CUDA error */

void plasma_note_cuda_error(void)
{
    cudaError_t e = cudaGetLastError();
    /* an allocation that failed is reported by the caller's return code */
    if (e != cudaSuccess && e != cudaErrorMemoryAllocation && plasma_cuda_error_g == 0)
        plasma_cuda_error_g = (int)e;
}

int plasma_take_cuda_error(void)
{
    plasma_note_cuda_error();
    int e = plasma_cuda_error_g;
    plasma_cuda_error_g = 0;
    return e;
}

plasma_context_t *plasma_context_self(void)
{
    return plasma_initialized_g ? &plasma_context_g : NULL;
}

static void context_defaults(plasma_context_t *c)
{
    memset(c, 0, sizeof(*c));
    c->tuning = PlasmaEnabled;
    c->nb = 256;
    c->ib = 64;
    c->inplace_outplace = PlasmaOutplace;
    c->max_threads = 1;
    c->max_panel_threads = 1;
    c->householder_mode = PlasmaFlatHouseholder;
    c->mixed_mode = PlasmaFactorFP32;
    c->refinement = PlasmaRefineIR;
    c->lookahead = 1;
    c->next_call = 1;
}

int plasma_init(void)
{
    if (plasma_initialized_g)
        return PlasmaErrorNotInitialized;

    plasma_context_t *c = &plasma_context_g;
    context_defaults(c);
    c->device = plasma_device_request_g;

    /* The factorization of a matrix that is still arriving keeps about 16
     * streams busy at once, several of them waiting on uploads; with the
     * driver's default of 8 hardware queues, streams share queues and a
     * wait at the head of one holds up the critical stream behind it.  The
     * setting takes effect when this call creates the CUDA context (an
     * application that created it earlier sets the variable itself). */
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        /* Host-only mode: lets argument checking and descriptor arithmetic
         * be exercised on machines without a GPU.  Every routine that would
         * touch the device returns PlasmaErrorEnvironment instead. */
        const char *env = getenv("PLASMA_ALLOW_NO_DEVICE");
        if (env && env[0] == '1') {
            c->device = -1;
            plasma_initialized_g = 1;
            return PlasmaSuccess;
        }
        plasma_error("no CUDA device available");
        return PlasmaErrorEnvironment;
    }
    if (c->device < 0 || c->device >= ndev) {
        plasma_error("invalid CUDA device");
        return PlasmaErrorIllegalValue;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        plasma_error("cudaSetDevice() failed");
        return PlasmaErrorEnvironment;
    }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount,
                           c->device);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)
            != cudaSuccess) {
        plasma_error("cudaStreamCreate() failed");
        return PlasmaErrorEnvironment;
    }
    c->stream = c->own_stream;
    /* aux[0]: critical path and aux[2]: uploads (highest priority: the
     * conversion of arriving columns gates the factorization), the others
     * (bulk and column-group updates) at the lowest priority */
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (int i = 0; i < PLASMA_NUM_STREAMS; i++)
        cudaStreamCreateWithPriority(&c->aux[i], cudaStreamNonBlocking,
                                     i == 0 || i == PLASMA_STREAM_COPY ? prio_hi : prio_lo);
    for (int i = 0; i < PLASMA_STAGE_STREAMS; i++) {
        cudaStreamCreateWithFlags(&c->stage[i], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&c->ev_stage[i], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&c->ev_stage_in, cudaEventDisableTiming);
    for (int i = 0; i < 8; i++)
        cudaEventCreateWithFlags(&c->ev[i], cudaEventDisableTiming);
    for (int i = 0; i < PLASMA_MAX_GROUPS; i++)
        cudaEventCreateWithFlags(&c->ev_group[i], cudaEventDisableTiming);
    if (cudaMalloc((void **)&c->dstat, sizeof(plasma_devstat_t)) != cudaSuccess ||
        cudaMalloc((void **)&c->dquiet, sizeof(plasma_devstat_t)) != cudaSuccess ||
        cudaMallocHost((void **)&c->hstat, sizeof(plasma_devstat_t)) != cudaSuccess) {
        plasma_error("cannot allocate the device status word");
        return PlasmaErrorOutOfMemory;
    }
    cudaMemset(c->dstat, 0, sizeof(plasma_devstat_t));
    cudaMemset(c->dquiet, 0, sizeof(plasma_devstat_t));
    cudaDeviceSynchronize();
    plasma_initialized_g = 1;
    return PlasmaSuccess;
}

int plasma_finalize(void)
{
    if (!plasma_initialized_g)
        return PlasmaErrorNotInitialized;
    plasma_context_t *c = &plasma_context_g;
    if (c->device < 0) {
        memset(c, 0, sizeof(*c));
        plasma_initialized_g = 0;
        return PlasmaSuccess;
    }
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    for (int i = 0; i < PLASMA_SCRATCH_SLOTS; i++)
        if (c->scratch[i]) cudaFree(c->scratch[i]);
    for (int i = 0; i < 8; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (int i = 0; i < PLASMA_MAX_GROUPS; i++)
        if (c->ev_group[i]) cudaEventDestroy(c->ev_group[i]);
    if (c->sweep_sync) cudaFree(c->sweep_sync);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->dstat) cudaFree(c->dstat);
    if (c->dquiet) cudaFree(c->dquiet);
    if (c->hstat) cudaFreeHost(c->hstat);
    for (int i = 0; i < PLASMA_NUM_STREAMS; i++)
        if (c->aux[i]) cudaStreamDestroy(c->aux[i]);
    for (int i = 0; i < PLASMA_STAGE_STREAMS; i++) {
        if (c->stage[i]) cudaStreamDestroy(c->stage[i]);
        if (c->ev_stage[i]) cudaEventDestroy(c->ev_stage[i]);
    }
    if (c->ev_stage_in) cudaEventDestroy(c->ev_stage_in);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    memset(c, 0, sizeof(*c));
    plasma_initialized_g = 0;
    return PlasmaSuccess;
}

int plasma_set(plasma_enum_t param, int value)
{
    if (param == PlasmaDevice && !plasma_initialized_g) {
        /* the device is chosen before plasma_init() */
        if (value < 0) return PlasmaErrorIllegalValue;
        plasma_device_request_g = value;
        return PlasmaSuccess;
    }
    if (!plasma_initialized_g)
        return PlasmaErrorNotInitialized;
    plasma_context_t *c = &plasma_context_g;

    switch (param) {
    case PlasmaTuning:
        if (value != PlasmaEnabled && value != PlasmaDisabled) {
            plasma_error("invalid tuning flag");
            return PlasmaErrorIllegalValue;
        }
        c->tuning = value;
        break;
    case PlasmaNb:
        if (value <= 0) {
            plasma_error("invalid tile size");
            return PlasmaErrorIllegalValue;
        }
        c->nb = value;
        break;
    case PlasmaIb:
        if (value <= 0) {
            plasma_error("invalid inner block size");
            return PlasmaErrorIllegalValue;
        }
        c->ib = value;
        break;
    case PlasmaNumPanelThreads:
        if (value <= 0) {
            plasma_error("invalid number of panel threads");
            return PlasmaErrorIllegalValue;
        }
        c->max_panel_threads = value;
        break;
    case PlasmaHouseholderMode:
        if (value != PlasmaFlatHouseholder && value != PlasmaTreeHouseholder) {
            plasma_error("invalid Householder mode");
            return PlasmaErrorIllegalValue;
        }
        c->householder_mode = value;
        break;
    case PlasmaMixedPrecisionMode:
        if (value < PlasmaFactorFP32 || value > PlasmaFactorAuto) {
            plasma_error("invalid mixed-precision mode");
            return PlasmaErrorIllegalValue;
        }
        c->mixed_mode = value;
        break;
    case PlasmaRefinement:
        if (value < PlasmaRefineIR || value > PlasmaRefineAuto) {
            plasma_error("invalid refinement scheme");
            return PlasmaErrorIllegalValue;
        }
        c->refinement = value;
        break;
    case PlasmaLookahead:
        if (value < 0) {
            plasma_error("invalid look-ahead depth");
            return PlasmaErrorIllegalValue;
        }
        c->lookahead = value;
        break;
    case PlasmaDevice:
        plasma_error("the device can only be set before plasma_init()");
        return PlasmaErrorIllegalValue;
    default:
        plasma_error("unknown parameter");
        return PlasmaErrorIllegalValue;
    }
    return PlasmaSuccess;
}

int plasma_get(plasma_enum_t param, int *value)
{
    if (!plasma_initialized_g)
        return PlasmaErrorNotInitialized;
    plasma_context_t *c = &plasma_context_g;
    switch (param) {
    case PlasmaTuning:             *value = c->tuning;            break;
    case PlasmaNb:                 *value = c->nb;                break;
    case PlasmaIb:                 *value = c->ib;                break;
    case PlasmaNumPanelThreads:    *value = c->max_panel_threads; break;
    case PlasmaHouseholderMode:    *value = c->householder_mode;  break;
    case PlasmaMixedPrecisionMode: *value = c->mixed_mode;        break;
    case PlasmaRefinement:         *value = c->refinement;        break;
    case PlasmaLookahead:          *value = c->lookahead;         break;
    case PlasmaDevice:             *value = c->device;            break;
    default:
        plasma_error("Unknown parameter");
        return PlasmaErrorIllegalValue;
    }
    return PlasmaSuccess;
}

void plasma_version(int *major, int *minor, int *micro)
{
    *major = PLASMA_VERSION_MAJOR;
    *minor = PLASMA_VERSION_MINOR;
    *micro = PLASMA_VERSION_PATCH;
}

int plasma_set_stream(void *stream)
{
    if (!plasma_initialized_g)
        return PlasmaErrorNotInitialized;
    plasma_context_g.stream = stream ? (cudaStream_t)stream
                                     : plasma_context_g.own_stream;
    return PlasmaSuccess;
}

void *plasma_get_stream(void)
{
    if (!plasma_initialized_g)
        return NULL;
    return (void *)plasma_context_g.stream;
}

long long plasma_kernel_launches(void)
{
    return plasma_launch_count_g;
}

long long plasma_device_allocations(void)
{
    return plasma_alloc_count_g;
}

int plasma_call_begin(plasma_context_t *c, plasma_sequence_t *sequence,
                      plasma_request_t *request)
{
    int id = c->next_call++;
    if (c->next_call >= PLASMA_MAX_PENDING_CALLS)
        c->next_call = 1;
    c->pending[id] = request;
    c->pending_seq[id] = sequence;
    return id;
}

void *plasma_scratch(plasma_context_t *c, int slot, size_t bytes)
{
    if (bytes <= c->scratch_bytes[slot])
        return c->scratch[slot];
    if (c->scratch[slot]) {
        /* growing: wait for every user of the old buffer */
        cudaStreamSynchronize(c->stream);
        for (int i = 0; i < PLASMA_NUM_STREAMS; i++)
            cudaStreamSynchronize(c->aux[i]);
        cudaFree(c->scratch[slot]);
        c->scratch[slot] = NULL;
        c->scratch_bytes[slot] = 0;
    }
    size_t want = bytes + bytes / 8 + (1u << 20);
    plasma_note_cuda_error();
    plasma_alloc_count_g++;
    if (cudaMalloc(&c->scratch[slot], want) != cudaSuccess) {
        plasma_note_cuda_error();
        c->scratch[slot] = NULL;
        return NULL;
    }
    c->scratch_bytes[slot] = want;
    return c->scratch[slot];
}

void *plasma_pinned(plasma_context_t *c, size_t bytes)
{
    if (bytes <= c->pinned_bytes)
        return c->pinned;
    if (c->pinned) {
        cudaStreamSynchronize(c->stream);
        for (int i = 0; i < PLASMA_STAGE_STREAMS; i++)
            cudaStreamSynchronize(c->stage[i]);
        cudaFreeHost(c->pinned);
        c->pinned = NULL;
        c->pinned_bytes = 0;
    }
    plasma_note_cuda_error();
    plasma_alloc_count_g++;
    if (cudaMallocHost(&c->pinned, bytes) != cudaSuccess) {
        cudaGetLastError();            /* the callers fall back; not an error */
        c->pinned = NULL;
        return NULL;
    }
    c->pinned_bytes = bytes;
    return c->pinned;
}

int plasma_is_pageable(const void *p)
{
    struct cudaPointerAttributes attr;
    if (p == NULL)
        return 0;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return attr.type == cudaMemoryTypeUnregistered;
}

int plasma_is_device_pointer(const void *p)
{
    struct cudaPointerAttributes attr;
    if (p == NULL)
        return 0;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return attr.type == cudaMemoryTypeDevice ||
           attr.type == cudaMemoryTypeManaged;
}

const char *plasma_strerror(int code)
{
    switch (code) {
    case PlasmaSuccess:             return "success";
    case PlasmaErrorNotInitialized: return "PLASMA not initialized";
    case PlasmaErrorNotSupported:   return "not supported";
    case PlasmaErrorIllegalValue:   return "illegal value";
    case PlasmaErrorOutOfMemory:    return "out of memory";
    case PlasmaErrorNullParameter:  return "NULL parameter";
    case PlasmaErrorInternal:       return "internal error";
    case PlasmaErrorSequence:       return "sequence error";
    case PlasmaErrorComponent:      return "component error";
    case PlasmaErrorEnvironment:    return "environment error";
    default:
        return code > 0 ? "matrix not positive definite (leading minor)"
                        : "illegal argument";
    }
}

/* Allocates the ready flags of one-launch sweeps with factor A; 0 when A's
 * tiles admit no one-launch sweep or the allocation fails. */
int plasma_sweep_reserve(plasma_context_t *c, plasma_desc_t A)
{
    int sb = plasma_cuda_trsv_block(A);
    if (sb == 0)
        return 0;
    size_t need = plasma_cuda_trsv_scratch_bytes(A);
    if (need > c->sweep_sync_bytes) {
        if (c->sweep_sync) {
            cudaStreamSynchronize(c->stream);
            cudaFree(c->sweep_sync);
        }
        c->sweep_sync = NULL;
        c->sweep_sync_bytes = 0;
        plasma_note_cuda_error();
        plasma_alloc_count_g++;
        if (cudaMalloc(&c->sweep_sync, need) != cudaSuccess) {
            plasma_note_cuda_error();
            return 0;
        }
        cudaMemsetAsync(c->sweep_sync, 0, need, c->stream);
        c->sweep_sync_bytes = need;
    }
    return 1;
}

int plasma_sweep(plasma_context_t *c, plasma_enum_t uplo, int backward,
                 plasma_desc_t A, const void *W, void *vec)
{
    if (!plasma_sweep_reserve(c, A))
        return 0;
    /* epochs are non-zero and change with every sweep */
    if (++c->sweep_epoch <= 0)
        c->sweep_epoch = 1;
    return plasma_cuda_trsv(c->stream, c->dstat, uplo, backward, A, W, vec,
                            c->sweep_sync, c->sweep_epoch, c->num_sms);
}

/* The multi-column one-launch sweep (up to 16 columns of the tile matrix B)
 * with the context's ready flags and a fresh epoch; 0 when not launched. */
int plasma_sweep_rows(plasma_context_t *c, plasma_enum_t uplo, int backward,
                      plasma_desc_t A, const void *W, plasma_desc_t B, int c0, int ncols)
{
    if (!plasma_sweep_reserve(c, A))
        return 0;
    if (++c->sweep_epoch <= 0)
        c->sweep_epoch = 1;
    return plasma_cuda_trsm_rows(c->stream, c->dstat, uplo, backward, A, W, B, c0, ncols,
                                 c->sweep_sync, c->sweep_epoch, c->num_sms);
}

/* A descriptor over a scratch slot that the context keeps between calls
 * (the LAPACK-layout drivers' tile copies): no allocation once the slot is
 * large enough, storage zeroed on the context stream.  type = PlasmaGeneral
 * or the uplo of a packed triangle.  The descriptor must not be destroyed. */
int plasma_desc_kept(plasma_context_t *c, int slot, plasma_enum_t precision,
                     plasma_enum_t type, int nb, int m, int n, plasma_desc_t *A)
{
    if (c->device < 0) {
        plasma_error("no CUDA device");
        return PlasmaErrorEnvironment;
    }
    const size_t mt = (size_t)(m + nb - 1) / nb, nt = (size_t)(n + nb - 1) / nb;
    const size_t tiles = type == PlasmaGeneral ? mt * nt : nt * (nt + 1) / 2;
    const size_t bytes = tiles * nb * nb * plasma_element_size(precision);
    void *buf = plasma_scratch(c, slot, bytes > 0 ? bytes : 16);
    if (buf == NULL)
        return PlasmaErrorOutOfMemory;
    int rc = type == PlasmaGeneral
                 ? plasma_desc_general_init(precision, buf, nb, nb, m, n, 0, 0, m, n, A)
                 : plasma_desc_triangular_init(precision, type, buf, nb, nb, m, n, 0, 0,
                                               m, n, A);
    if (rc != PlasmaSuccess)
        return rc;
    if (plasma_desc_storage_bytes(*A) > bytes)
        return PlasmaErrorInternal;
    cudaMemsetAsync(buf, 0, plasma_desc_storage_bytes(*A), c->stream);
    return PlasmaSuccess;
}
