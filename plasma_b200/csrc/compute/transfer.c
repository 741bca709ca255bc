/*
 * transfer.c -- LAPACK-layout <-> tile-layout conversion, host or device
 * source.
 *
 * plasma_omp_{d,s}{ge2desc,desc2ge,tr2desc,desc2tr} follow the reference's
 * compute/zge2desc.c:27-68 (argument checks, then one lacpy per tile,
 * compute/pzge2desc.c:22-56, pztr2desc.c:22-51).  The user array may live on
 * the host (it is staged through a device column-major buffer; pageable
 * host memory also goes through the page-locked slots of
 * control/staging.c) or on the device (packed directly by the kernel).
 */
#include "../internal.h"

#include <cuda_runtime_api.h>

/* Host <-> device copy of the part of a column-major array that a
 * descriptor view covers: all of it for PlasmaGeneral, or only the tile
 * columns' triangle part (from the diagonal tile down, or up to it) for
 * PlasmaLower / PlasmaUpper -- half the PCIe traffic for potrf/posv. */
static void copy_region(plasma_context_t *plasma, void *dst, size_t ldd,
                        const void *src, size_t lds, int rows, int cols,
                        int nb, plasma_enum_t uplo, size_t elem,
                        enum cudaMemcpyKind kind)
{
    if (rows <= 0 || cols <= 0)
        return;
    const void *host = kind == cudaMemcpyHostToDevice ? src : dst;
    if (plasma_is_pageable(host)) {
        plasma_stage_begin(plasma, plasma->stream);
        if (uplo != PlasmaLower && uplo != PlasmaUpper) {
            plasma_stage_copy(plasma, dst, ldd * elem, src, lds * elem, (size_t)rows * elem,
                              (size_t)cols, kind);
        } else {
            for (int c0 = 0; c0 < cols; c0 += nb) {
                int w = cols - c0 < nb ? cols - c0 : nb;
                int r0 = uplo == PlasmaLower ? (c0 < rows ? c0 : rows) : 0;
                int r1 = uplo == PlasmaLower ? rows : (c0 + nb < rows ? c0 + nb : rows);
                if (r1 > r0)
                    plasma_stage_copy(plasma, (char *)dst + ((size_t)c0 * ldd + r0) * elem,
                                      ldd * elem,
                                      (const char *)src + ((size_t)c0 * lds + r0) * elem,
                                      lds * elem, (size_t)(r1 - r0) * elem, (size_t)w, kind);
            }
        }
        plasma_stage_join(plasma, plasma->stream);
        return;
    }
    if (uplo != PlasmaLower && uplo != PlasmaUpper) {
        cudaMemcpy2DAsync(dst, ldd * elem, src, lds * elem,
                          (size_t)rows * elem, (size_t)cols, kind,
                          plasma->stream);
        return;
    }
    for (int c0 = 0; c0 < cols; c0 += nb) {
        int w = cols - c0 < nb ? cols - c0 : nb;
        int r0 = uplo == PlasmaLower ? (c0 < rows ? c0 : rows) : 0;
        int r1 = uplo == PlasmaLower ? rows : (c0 + nb < rows ? c0 + nb : rows);
        if (r1 <= r0)
            continue;
        cudaMemcpy2DAsync((char *)dst + ((size_t)c0 * ldd + r0) * elem,
                          ldd * elem,
                          (const char *)src + ((size_t)c0 * lds + r0) * elem,
                          lds * elem, (size_t)(r1 - r0) * elem, (size_t)w,
                          kind, plasma->stream);
    }
}

static int check_xfer(plasma_context_t *plasma, const void *pA, int lda,
                      plasma_desc_t A, plasma_sequence_t *sequence,
                      plasma_request_t *request)
{
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return 0;
    }
    if (plasma_desc_check(A) != PlasmaSuccess) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (pA == NULL) {
        plasma_error("NULL A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return 0;
    }
    if (lda < A.m) {
        plasma_error("illegal value of lda");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return 0;
    }
    if (plasma->device < 0) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return 0;
    }
    return sequence->status == PlasmaSuccess;
}

void plasma_omp_Xlapack2desc(const void *pA, int lda, plasma_desc_t A,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_xfer(plasma, pA, lda, A, sequence, request))
        return;
    if (A.m == 0 || A.n == 0)
        return;
    size_t elem = plasma_element_size(A.precision);
    const void *src = pA;
    int ld = lda;
    if (!plasma_is_device_pointer(pA)) {
        /* the staged copy starts at the view's tile-aligned origin */
        int rows = A.m + A.i % A.mb, cols = A.n + A.j % A.nb;
        ld = rows;
        void *buf = plasma_scratch(plasma, PLASMA_SLOT_STAGING,
                                   (size_t)ld * (size_t)cols * elem);
        if (buf == NULL) {
            plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
            return;
        }
        copy_region(plasma, buf, (size_t)ld, pA, (size_t)lda, rows, cols,
                    A.nb, uplo, elem, cudaMemcpyHostToDevice);
        src = buf;
    }
    plasma_cuda_lapack_to_tile(plasma->stream, plasma->dstat, A, uplo, src, ld);
}

void plasma_omp_Xdesc2lapack(plasma_desc_t A, void *pA, int lda,
                             plasma_enum_t uplo, plasma_sequence_t *sequence,
                             plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_xfer(plasma, pA, lda, A, sequence, request))
        return;
    if (A.m == 0 || A.n == 0)
        return;
    if (plasma_is_device_pointer(pA)) {
        plasma_cuda_tile_to_lapack(plasma->stream, plasma->dstat, A, uplo,
                                   pA, lda);
        return;
    }
    size_t elem = plasma_element_size(A.precision);
    int rows = A.m + A.i % A.mb, cols = A.n + A.j % A.nb;
    int ld = rows;
    void *buf = plasma_scratch(plasma, PLASMA_SLOT_STAGING,
                               (size_t)ld * (size_t)cols * elem);
    if (buf == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_cuda_tile_to_lapack(plasma->stream, plasma->dstat, A, uplo, buf, ld);
    copy_region(plasma, pA, (size_t)lda, buf, (size_t)ld, rows, cols, A.nb,
                uplo, elem, cudaMemcpyDeviceToHost);
    cudaStreamSynchronize(plasma->stream);
}

/* The upper triangle of the column-major pA into the lower descriptor A,
 * transposed (A = U^T), and back: the LAPACK-layout drivers factor an
 * upper-stored matrix through lower tiles.  Host arrays are staged through
 * the device buffer (upper triangle only). */
void plasma_omp_Xlapack2desc_t(const void *pA, int lda, plasma_desc_t A,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_xfer(plasma, pA, lda, A, sequence, request))
        return;
    if (A.m == 0 || A.n == 0)
        return;
    size_t elem = plasma_element_size(A.precision);
    const void *src = pA;
    int ld = lda;
    if (!plasma_is_device_pointer(pA)) {
        ld = A.m;
        void *buf = plasma_scratch(plasma, PLASMA_SLOT_STAGING,
                                   (size_t)ld * (size_t)A.n * elem);
        if (buf == NULL) {
            plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
            return;
        }
        copy_region(plasma, buf, (size_t)ld, pA, (size_t)lda, A.m, A.n, A.nb,
                    PlasmaUpper, elem, cudaMemcpyHostToDevice);
        src = buf;
    }
    plasma_cuda_lapack_to_tile_t(plasma->stream, plasma->dstat, A, src, ld);
}

void plasma_omp_Xdesc2lapack_t(plasma_desc_t A, void *pA, int lda,
                               plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (!check_xfer(plasma, pA, lda, A, sequence, request))
        return;
    if (A.m == 0 || A.n == 0)
        return;
    if (plasma_is_device_pointer(pA)) {
        plasma_cuda_tile_to_lapack_t(plasma->stream, plasma->dstat, A, pA, lda);
        return;
    }
    size_t elem = plasma_element_size(A.precision);
    int ld = A.m;
    void *buf = plasma_scratch(plasma, PLASMA_SLOT_STAGING, (size_t)ld * (size_t)A.n * elem);
    if (buf == NULL) {
        plasma_request_fail(sequence, request, PlasmaErrorOutOfMemory);
        return;
    }
    plasma_cuda_tile_to_lapack_t(plasma->stream, plasma->dstat, A, buf, ld);
    copy_region(plasma, pA, (size_t)lda, buf, (size_t)ld, A.m, A.n, A.nb, PlasmaUpper, elem,
                cudaMemcpyDeviceToHost);
    cudaStreamSynchronize(plasma->stream);
}

void plasma_omp_dge2desc(double *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xlapack2desc(pA, lda, A, PlasmaGeneral, sequence, request);
}

void plasma_omp_ddesc2ge(plasma_desc_t A, double *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2lapack(A, pA, lda, PlasmaGeneral, sequence, request);
}

void plasma_omp_dtr2desc(double *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xlapack2desc(pA, lda, A, A.type, sequence, request);
}

void plasma_omp_ddesc2tr(plasma_desc_t A, double *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2lapack(A, pA, lda, A.type, sequence, request);
}

void plasma_omp_sge2desc(float *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xlapack2desc(pA, lda, A, PlasmaGeneral, sequence, request);
}

void plasma_omp_sdesc2ge(plasma_desc_t A, float *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2lapack(A, pA, lda, PlasmaGeneral, sequence, request);
}

void plasma_omp_str2desc(float *pA, int lda, plasma_desc_t A,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xlapack2desc(pA, lda, A, A.type, sequence, request);
}

void plasma_omp_sdesc2tr(plasma_desc_t A, float *pA, int lda,
                         plasma_sequence_t *sequence, plasma_request_t *request)
{
    plasma_omp_Xdesc2lapack(A, pA, lda, A.type, sequence, request);
}
