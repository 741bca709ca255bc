/*
 * staging.c -- host <-> device copies of column-major blocks whose host side
 * is pageable memory (what a C caller's malloc'd arrays are).
 *
 * The reference's LAPACK-layout drivers translate the user's arrays into
 * tiles and back in host memory (compute/zpotrf.c:134-140,
 * plasma_omp_ztr2desc / plasma_omp_zdesc2tr).  Here those arrays cross
 * PCIe, and cudaMemcpy*Async from pageable memory first waits for its
 * stream to drain and then copies through the driver's own small buffers
 * (about 11 GB/s on the B200 hosts, against 55 GB/s from page-locked
 * memory).  So a pageable block goes through PLASMA_STAGE_STREAMS
 * page-locked slots of STAGE_SLOT_BYTES: per chunk of whole columns, a host
 * function on a staging stream copies the chunk between the user's array
 * and the stream's slot (OpenMP threads, streaming stores), and
 * cudaMemcpy2DAsync moves the slot to or from the device.  Chunks go round
 * the staging streams, so host copies overlap transfers; a slot is
 * rewritten only after the transfer that read it, which precedes the
 * rewrite on the slot's own stream.
 *
 *   plasma_stage_begin(plasma, s)   staging streams start after s's work
 *   plasma_stage_copy(...)          enqueue one block (no ordering with s)
 *   plasma_stage_join(plasma, s)    s waits for everything staged so far
 *
 * plasma_copy_2d does the three for one block, and copies page-locked or
 * device memory directly on the stream.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#define STAGE_SLOT_BYTES ((size_t)32 << 20)
#define STAGE_SEGMENT    ((size_t)64 << 10)     /* bytes one thread copies */

typedef struct {
    char *dst;
    size_t dpitch;
    const char *src;
    size_t spitch;
    size_t width;        /* bytes per column */
    size_t height;       /* columns          */
} stage_job_t;

#if defined(__x86_64__)
/* Streaming stores: the destination line is written without being read
 * first, so the copy moves each byte through memory once, next to the
 * transfer engine's reads of the other slots. */
__attribute__((target("avx2")))
static void copy_bytes_stream(char *d, const char *s, size_t bytes)
{
    size_t r = 0;
    while (r < bytes && ((uintptr_t)(d + r) & 31) != 0) {
        d[r] = s[r];
        r++;
    }
    for (; r + 64 <= bytes; r += 64) {
        __m256i x0 = _mm256_loadu_si256((const __m256i *)(s + r));
        __m256i x1 = _mm256_loadu_si256((const __m256i *)(s + r + 32));
        _mm256_stream_si256((__m256i *)(d + r), x0);
        _mm256_stream_si256((__m256i *)(d + r + 32), x1);
    }
    for (; r < bytes; r++)
        d[r] = s[r];
    _mm_sfence();       /* this thread's streaming stores before the transfer */
}
#endif

static void copy_bytes(char *d, const char *s, size_t bytes)
{
#if defined(__x86_64__)
    if (__builtin_cpu_supports("avx2")) {
        copy_bytes_stream(d, s, bytes);
        return;
    }
#endif
    memcpy(d, s, bytes);
}

/* One chunk between the user's array and a slot, split into segments of
 * STAGE_SEGMENT bytes of one column each, spread over the OpenMP threads;
 * frees its job. */
static void CUDART_CB stage_run(void *p)
{
    stage_job_t *j = (stage_job_t *)p;
    const size_t segs = (j->width + STAGE_SEGMENT - 1) / STAGE_SEGMENT;
    const long total = (long)(segs * j->height);
    #pragma omp parallel for schedule(static)
    for (long t = 0; t < total; t++) {
        const size_t c = (size_t)t / segs;
        const size_t o = ((size_t)t % segs) * STAGE_SEGMENT;
        const size_t b = j->width - o < STAGE_SEGMENT ? j->width - o : STAGE_SEGMENT;
        copy_bytes(j->dst + c * j->dpitch + o, j->src + c * j->spitch + o, b);
    }
    free(j);
}

void plasma_stage_begin(plasma_context_t *plasma, cudaStream_t s)
{
    cudaEventRecord(plasma->ev_stage_in, s);
    for (int i = 0; i < PLASMA_STAGE_STREAMS; i++)
        cudaStreamWaitEvent(plasma->stage[i], plasma->ev_stage_in, 0);
}

void plasma_stage_join(plasma_context_t *plasma, cudaStream_t s)
{
    for (int i = 0; i < PLASMA_STAGE_STREAMS; i++) {
        cudaEventRecord(plasma->ev_stage[i], plasma->stage[i]);
        cudaStreamWaitEvent(s, plasma->ev_stage[i], 0);
    }
}

void plasma_stage_copy(plasma_context_t *plasma, void *dst, size_t dpitch, const void *src,
                       size_t spitch, size_t width, size_t height, enum cudaMemcpyKind kind)
{
    if (width == 0 || height == 0)
        return;
    char *ring = width <= STAGE_SLOT_BYTES
                     ? (char *)plasma_pinned(plasma, PLASMA_STAGE_STREAMS * STAGE_SLOT_BYTES)
                     : NULL;
    if (ring == NULL) {
        /* no slots (or columns longer than one): the driver's own path */
        cudaStream_t s = plasma->stage[plasma->stage_next++ % PLASMA_STAGE_STREAMS];
        cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, s);
        return;
    }
    const size_t per = STAGE_SLOT_BYTES / width;      /* columns per chunk */
    for (size_t c0 = 0; c0 < height; c0 += per) {
        const size_t h = height - c0 < per ? height - c0 : per;
        const int i = plasma->stage_next++ % PLASMA_STAGE_STREAMS;
        cudaStream_t s = plasma->stage[i];
        char *slot = ring + (size_t)i * STAGE_SLOT_BYTES;
        char *d = (char *)dst + c0 * dpitch;
        const char *sp = (const char *)src + c0 * spitch;
        stage_job_t *j = (stage_job_t *)malloc(sizeof(stage_job_t));
        if (j == NULL) {
            /* the driver's own path, in order on the same stream */
            cudaMemcpy2DAsync(d, dpitch, sp, spitch, width, h, kind, s);
            continue;
        }
        j->width = width;
        j->height = h;
        if (kind == cudaMemcpyHostToDevice) {
            j->dst = slot;
            j->dpitch = width;
            j->src = sp;
            j->spitch = spitch;
            cudaLaunchHostFunc(s, stage_run, j);
            cudaMemcpy2DAsync(d, dpitch, slot, width, width, h, kind, s);
        } else {
            j->dst = d;
            j->dpitch = dpitch;
            j->src = slot;
            j->spitch = width;
            cudaMemcpy2DAsync(slot, width, sp, spitch, width, h, kind, s);
            cudaLaunchHostFunc(s, stage_run, j);
        }
    }
}

void plasma_copy_2d(plasma_context_t *plasma, cudaStream_t s, void *dst, size_t dpitch,
                    const void *src, size_t spitch, size_t width, size_t height,
                    enum cudaMemcpyKind kind, int pageable)
{
    if (width == 0 || height == 0)
        return;
    if (pageable) {
        plasma_stage_begin(plasma, s);
        plasma_stage_copy(plasma, dst, dpitch, src, spitch, width, height, kind);
        plasma_stage_join(plasma, s);
        return;
    }
    cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, s);
}
