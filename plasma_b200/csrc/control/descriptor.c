/*
 * descriptor.c -- tile descriptors.
 *
 * Shape arithmetic and checks follow the reference's control/descriptor.c
 * (general_init :134-175, triangular_init :216-264, general_check :283-319,
 * view :374-397; band init and check :178-213, :321-369) because the region
 * offsets A21/A12/A22 and the band tile counts define the storage format
 * shared with callers.  Storage made by the *_create routines is device
 * memory of the context's GPU (the reference uses malloc, :40 and :108-113),
 * zero-filled so that padding never holds stale values.
 */
#include "../internal.h"

#include <cuda_runtime_api.h>
#include <string.h>

size_t plasma_desc_storage_bytes(plasma_desc_t A)
{
    size_t elems;
    if (A.type == PlasmaGeneral || A.type == PlasmaGeneralBand) {
        elems = (size_t)A.gm * A.gn;
    }
    else {
        size_t lm1 = (size_t)(A.gm / A.mb);
        size_t ln1 = (size_t)(A.gn / A.nb);
        size_t mnt = (ln1 * (1 + lm1)) / 2;
        elems = mnt * A.mb * A.nb + (size_t)A.gm * (A.gn % A.nb);
    }
    return elems * plasma_element_size(A.precision);
}

static int desc_alloc(plasma_desc_t *A)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma->device < 0) {
        plasma_error("no CUDA device");
        return PlasmaErrorEnvironment;
    }
    size_t bytes = plasma_desc_storage_bytes(*A);
    A->matrix = NULL;
    if (bytes == 0)
        bytes = 16;
    plasma_note_cuda_error();
    plasma_alloc_count_g++;
    if (cudaMalloc(&A->matrix, bytes) != cudaSuccess) {
        plasma_note_cuda_error();
        A->matrix = NULL;
        plasma_error("cudaMalloc() failed");
        return PlasmaErrorOutOfMemory;
    }
    cudaMemsetAsync(A->matrix, 0, bytes, plasma->stream);
    return PlasmaSuccess;
}

int plasma_desc_general_create(plasma_enum_t precision, int mb, int nb,
                               int lm, int ln, int i, int j, int m, int n,
                               plasma_desc_t *A)
{
    if (plasma_context_self() == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    int retval = plasma_desc_general_init(precision, NULL, mb, nb,
                                          lm, ln, i, j, m, n, A);
    if (retval != PlasmaSuccess)
        return retval;
    if (plasma_desc_check(*A) != PlasmaSuccess) {
        plasma_error("plasma_desc_check() failed");
        return PlasmaErrorIllegalValue;
    }
    return desc_alloc(A);
}

int plasma_desc_triangular_create(plasma_enum_t precision, plasma_enum_t uplo,
                                  int mb, int nb, int lm, int ln,
                                  int i, int j, int m, int n,
                                  plasma_desc_t *A)
{
    if (plasma_context_self() == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    int retval = plasma_desc_triangular_init(precision, uplo, NULL, mb, nb,
                                             lm, ln, i, j, m, n, A);
    if (retval != PlasmaSuccess)
        return retval;
    if (plasma_desc_check(*A) != PlasmaSuccess) {
        plasma_error("plasma_desc_check() failed");
        return PlasmaErrorIllegalValue;
    }
    return desc_alloc(A);
}

int plasma_desc_general_band_create(plasma_enum_t precision, plasma_enum_t uplo,
                                    int mb, int nb, int lm, int ln,
                                    int i, int j, int m, int n, int kl, int ku,
                                    plasma_desc_t *A)
{
    if (plasma_context_self() == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    int retval = plasma_desc_general_band_init(precision, uplo, NULL, mb, nb, lm, ln,
                                               i, j, m, n, kl, ku, A);
    if (retval != PlasmaSuccess)
        return retval;
    if (plasma_desc_check(*A) != PlasmaSuccess) {
        plasma_error("plasma_desc_check() failed");
        return PlasmaErrorIllegalValue;
    }
    return desc_alloc(A);
}

int plasma_desc_destroy(plasma_desc_t *A)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        return PlasmaErrorNotInitialized;
    }
    if (A->matrix) {
        /* kernels reading the storage may still be queued */
        cudaStreamSynchronize(plasma->stream);
        cudaFree(A->matrix);
    }
    A->matrix = NULL;
    return PlasmaSuccess;
}

static void set_view(plasma_desc_t *A, int i, int j, int m, int n)
{
    A->i = i;
    A->j = j;
    A->m = m;
    A->n = n;
    A->mt = (m == 0) ? 0 : (i + m - 1) / A->mb - i / A->mb + 1;
    A->nt = (n == 0) ? 0 : (j + n - 1) / A->nb - j / A->nb + 1;
}

int plasma_desc_general_init(plasma_enum_t precision, void *matrix,
                             int mb, int nb, int lm, int ln, int i, int j,
                             int m, int n, plasma_desc_t *A)
{
    memset(A, 0, sizeof(*A));
    A->type = PlasmaGeneral;
    A->precision = precision;
    A->matrix = matrix;
    A->mb = mb;
    A->nb = nb;
    A->gm = lm;
    A->gn = ln;
    if (mb <= 0 || nb <= 0) {
        /* let plasma_desc_check() report it */
        return PlasmaSuccess;
    }
    size_t full_rows = (size_t)(lm - lm % mb);
    size_t full_cols = (size_t)(ln - ln % nb);
    A->A21 = full_rows * full_cols;
    A->A12 = (size_t)(lm % mb) * full_cols + A->A21;
    A->A22 = full_rows * (size_t)(ln % nb) + A->A12;
    A->gmt = (lm + mb - 1) / mb;
    A->gnt = (ln + nb - 1) / nb;
    set_view(A, i, j, m, n);
    A->kl = m - 1;
    A->ku = n - 1;
    A->klt = A->mt;
    A->kut = A->nt;
    return PlasmaSuccess;
}

/* A general layout whose tile columns hold the band's tiles; the tile-row
 * counts of the band (reference control/descriptor.c:199-211):
 * klt = tiles on and below the diagonal, kut = on and above. */
int plasma_desc_general_band_init(plasma_enum_t precision, plasma_enum_t uplo,
                                  void *matrix, int mb, int nb, int lm, int ln,
                                  int i, int j, int m, int n, int kl, int ku,
                                  plasma_desc_t *A)
{
    int retval = plasma_desc_general_init(precision, matrix, mb, nb, lm, ln, i, j, m, n, A);
    if (retval != PlasmaSuccess)
        return retval;
    A->type = PlasmaGeneralBand;
    A->uplo = uplo;
    A->kl = kl;
    A->ku = ku;
    if (mb <= 0 || nb <= 0)
        return PlasmaSuccess;
    if (uplo == PlasmaGeneral) {
        A->klt = 1 + (i + kl + mb - 1) / mb - i / mb;
        A->kut = 1 + (i + ku + kl + nb - 1) / nb - i / nb;
    }
    else if (uplo == PlasmaUpper) {
        A->klt = 1;
        A->kut = 1 + (i + ku + nb - 1) / nb - i / nb;
    }
    else {
        A->klt = 1 + (i + kl + mb - 1) / mb - i / mb;
        A->kut = 1;
    }
    return PlasmaSuccess;
}

int plasma_desc_triangular_init(plasma_enum_t precision, plasma_enum_t uplo,
                                void *matrix, int mb, int nb, int lm, int ln,
                                int i, int j, int m, int n, plasma_desc_t *A)
{
    memset(A, 0, sizeof(*A));
    if (lm != ln)
        plasma_error("invalid lm or ln");
    A->type = uplo;
    A->precision = precision;
    A->matrix = matrix;
    A->mb = mb;
    A->nb = nb;
    A->gm = lm;
    A->gn = ln;
    if (mb <= 0 || nb <= 0)
        return PlasmaSuccess;
    size_t lm1 = (size_t)(lm / mb);
    size_t ln1 = (size_t)(ln / nb);
    size_t mnt = (ln1 * (1 + lm1)) / 2;
    A->A21 = (size_t)mb * nb * mnt;
    A->A12 = (size_t)mb * nb * mnt;
    A->A22 = (size_t)(lm - lm % mb) * (size_t)(ln % nb) + A->A12;
    A->gmt = (lm + mb - 1) / mb;
    A->gnt = (ln + nb - 1) / nb;
    set_view(A, i, j, m, n);
    A->kl = m - 1;
    A->ku = n - 1;
    A->klt = A->mt;
    A->kut = A->nt;
    return PlasmaSuccess;
}

int plasma_desc_check(plasma_desc_t A)
{
    if (A.type == PlasmaGeneral || A.type == PlasmaUpper ||
        A.type == PlasmaLower)
        return plasma_desc_general_check(A);
    if (A.type == PlasmaGeneralBand)
        return plasma_desc_general_band_check(A);
    plasma_error("invalid matrix type");
    return PlasmaErrorIllegalValue;
}

/* The reference's checks (control/descriptor.c:321-369), with the storage
 * rule the tile addressing relies on stated exactly: gm holds the
 * kut + klt - 1 tile rows of a band column and is a multiple of mb, and the
 * view starts on the diagonal (i = j). */
int plasma_desc_general_band_check(plasma_desc_t A)
{
    if (A.precision != PlasmaRealFloat && A.precision != PlasmaRealDouble &&
        A.precision != PlasmaComplexFloat &&
        A.precision != PlasmaComplexDouble) {
        plasma_error("invalid matrix type");
        return PlasmaErrorIllegalValue;
    }
    if (A.uplo != PlasmaGeneral && A.uplo != PlasmaUpper && A.uplo != PlasmaLower) {
        plasma_error("invalid band uplo");
        return PlasmaErrorIllegalValue;
    }
    if (A.mb <= 0 || A.nb <= 0) {
        plasma_error("negative tile dimension");
        return PlasmaErrorIllegalValue;
    }
    if (A.m < 0 || A.n < 0 || A.kl < 0 || A.ku < 0) {
        plasma_error("negative matrix dimension");
        return PlasmaErrorIllegalValue;
    }
    if (A.gn < A.n) {
        plasma_error("invalid leading column dimensions");
        return PlasmaErrorIllegalValue;
    }
    if (A.gm % A.mb != 0 || A.gm < A.mb * (A.kut + A.klt - 1)) {
        plasma_error("invalid leading row dimensions");
        return PlasmaErrorIllegalValue;
    }
    if (A.j > 0 && A.j >= A.gn) {
        plasma_error("beginning of the matrix out of bounds");
        return PlasmaErrorIllegalValue;
    }
    if (A.j + A.n > A.gn) {
        plasma_error("submatrix out of bounds");
        return PlasmaErrorIllegalValue;
    }
    if (A.i % A.mb != 0 || A.j % A.nb != 0 || A.i != A.j) {
        plasma_error("submatrix not aligned to a diagonal tile");
        return PlasmaErrorIllegalValue;
    }
    if (A.kl + 1 > A.m || A.ku + 1 > A.n) {
        plasma_error("band width larger than matrix dimension");
        return PlasmaErrorIllegalValue;
    }
    return PlasmaSuccess;
}

int plasma_desc_general_check(plasma_desc_t A)
{
    if (A.precision != PlasmaRealFloat && A.precision != PlasmaRealDouble &&
        A.precision != PlasmaComplexFloat &&
        A.precision != PlasmaComplexDouble) {
        plasma_error("invalid matrix type");
        return PlasmaErrorIllegalValue;
    }
    if (A.mb <= 0 || A.nb <= 0) {
        plasma_error("negative tile dimension");
        return PlasmaErrorIllegalValue;
    }
    if (A.m < 0 || A.n < 0) {
        plasma_error("negative matrix dimension");
        return PlasmaErrorIllegalValue;
    }
    if (A.gm < A.m || A.gn < A.n) {
        plasma_error("invalid leading dimensions");
        return PlasmaErrorIllegalValue;
    }
    if ((A.i > 0 && A.i >= A.gm) || (A.j > 0 && A.j >= A.gn)) {
        plasma_error("beginning of the matrix out of bounds");
        return PlasmaErrorIllegalValue;
    }
    if (A.i + A.m > A.gm || A.j + A.n > A.gn) {
        plasma_error("submatrix out of bounds");
        return PlasmaErrorIllegalValue;
    }
    if (A.i % A.mb != 0 || A.j % A.nb != 0) {
        plasma_error("submatrix not aligned to a tile");
        return PlasmaErrorIllegalValue;
    }
    return PlasmaSuccess;
}

plasma_desc_t plasma_desc_view(plasma_desc_t A, int i, int j, int m, int n)
{
    if (A.i + i + m > A.gm)
        plasma_fatal_error("rows out of bound");
    if (A.j + j + n > A.gn)
        plasma_fatal_error("columns out of bound");
    plasma_desc_t B = A;
    set_view(&B, A.i + i, A.j + j, m, n);
    return B;
}
