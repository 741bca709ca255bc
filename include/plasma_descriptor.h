/*
 * plasma_descriptor.h -- the tile matrix descriptor.
 *
 * The struct below keeps the reference's field order and meaning
 * (include/plasma_descriptor.h:40-76) because it is passed by value across the
 * C API.  The tile address arithmetic is the storage format itself and so
 * follows the same formulas (include/plasma_descriptor.h:93-151):
 *
 *   general  : tile (m,n) of the full-tile block A11 starts at
 *              mb*nb*(m + lm1*n) elements, lm1 = gm/mb;
 *   triangle : lower  tile (m,n), n <= m, at mb*nb*((m-n) + n*(2*lm1-n+1)/2),
 *              upper  tile (m,n), m <= n, at mb*nb*(m + n*(n+1)/2);
 *   ragged   : the last tile row (height gm%mb) lives in region A21, the last
 *              tile column (width gn%nb) in A12, the corner tile in A22;
 *   band     : tile (m,n) at the general position ((kut-1)+m-n, n) of a
 *              layout gm = mb*(kut+klt-1) rows high (:154-157).
 *
 * Each tile is column-major with leading dimension plasma_tile_mmain().
 *
 * GPU build: descriptors made by plasma_desc_*_create() own DEVICE memory
 * (cudaMalloc on the context's device); *_init() wraps memory the caller
 * owns, which must be device-accessible for the plasma_omp_* routines.  The
 * inline helpers are usable from host and device code.
 */
#ifndef PLASMA_DESCRIPTOR_H
#define PLASMA_DESCRIPTOR_H

#include "plasma_types.h"
#include "plasma_error.h"

#include <stddef.h>

#if defined(__CUDACC__)
#define PLASMA_HD __host__ __device__ __forceinline__
#else
#define PLASMA_HD static inline
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* matrix properties */
    plasma_enum_t type;      /* PlasmaGeneral, PlasmaLower, PlasmaUpper ... */
    plasma_enum_t uplo;      /* band descriptors only                       */
    plasma_enum_t precision; /* PlasmaRealDouble, PlasmaRealFloat ...       */

    /* storage and region offsets (in elements) */
    void  *matrix;
    size_t A21;
    size_t A12;
    size_t A22;

    /* tile shape */
    int mb;
    int nb;

    /* whole matrix */
    int gm;
    int gn;
    int gmt;
    int gnt;

    /* sub-matrix view */
    int i;
    int j;
    int m;
    int n;
    int mt;
    int nt;

    /* band parameters */
    int kl;
    int ku;
    int klt;
    int kut;
} plasma_desc_t;

PLASMA_HD size_t plasma_element_size(int type)
{
    return type == PlasmaRealDouble   ? 8 :
           type == PlasmaRealFloat    ? 4 :
           type == PlasmaComplexDouble ? 16 :
           type == PlasmaComplexFloat ? 8 :
           type == PlasmaInteger      ? sizeof(int) : 1;
}

/* Element offset of tile (m,n) of a general descriptor. */
PLASMA_HD size_t plasma_tile_offset_general(plasma_desc_t A, int m, int n)
{
    size_t mm = (size_t)(m + A.i / A.mb);
    size_t nn = (size_t)(n + A.j / A.nb);
    size_t lm1 = (size_t)(A.gm / A.mb);
    size_t ln1 = (size_t)(A.gn / A.nb);
    if (mm < lm1)
        return nn < ln1 ? (size_t)A.mb * A.nb * (mm + lm1 * nn)
                        : A.A12 + (size_t)A.mb * (A.gn % A.nb) * mm;
    return nn < ln1 ? A.A21 + (size_t)A.nb * (A.gm % A.mb) * nn
                    : A.A22;
}

/* Element offset of tile (m,n) of a packed triangular descriptor. */
PLASMA_HD size_t plasma_tile_offset_triangle(plasma_desc_t A, int m, int n)
{
    size_t mm = (size_t)(m + A.i / A.mb);
    size_t nn = (size_t)(n + A.j / A.nb);
    size_t lm1 = (size_t)(A.gm / A.mb);
    size_t ln1 = (size_t)(A.gn / A.nb);
    if (mm < lm1) {
        if (nn < ln1) {
            size_t t = A.type == PlasmaUpper
                     ? mm + (nn * (nn + 1)) / 2
                     : (mm - nn) + (nn * (2 * lm1 - (nn - 1))) / 2;
            return (size_t)A.mb * A.nb * t;
        }
        return A.A12 + (size_t)A.mb * (A.gn % A.nb) * mm;
    }
    return nn < ln1 ? A.A21 + (size_t)A.nb * (A.gm % A.mb) * nn
                    : A.A22;
}

/* Element offset of tile (m,n) of a band descriptor (type PlasmaGeneralBand,
 * reference include/plasma_descriptor.h:154-157): the tiles of the band of
 * tile column n are stored down column n of a general layout with gm/mb tile
 * rows, tile (m,n) at tile row (kut-1) + m - n.  The view starts on the
 * diagonal (i = j), and gm is a multiple of mb, so only the last tile column
 * can be narrow (region A12) -- plasma_desc_general_band_check. */
PLASMA_HD size_t plasma_tile_offset(plasma_desc_t A, int m, int n)
{
    if (A.type == PlasmaLower || A.type == PlasmaUpper)
        return plasma_tile_offset_triangle(A, m, n);
    /* band: the general formula at the stored tile row */
    const int row = A.type == PlasmaGeneralBand ? A.kut - 1 + m - n - A.i / A.mb : m;
    return plasma_tile_offset_general(A, row, n);
}

PLASMA_HD void *plasma_tile_addr(plasma_desc_t A, int m, int n)
{
    return (void *)((char *)A.matrix +
                    plasma_tile_offset(A, m, n) * plasma_element_size(A.precision));
}

/* Height of the tile stored at tile row k (its leading dimension). */
PLASMA_HD int plasma_tile_mmain(plasma_desc_t A, int k)
{
    /* with gm a multiple of mb every stored tile is mb rows high (no tile
     * row of height 0 exists); band descriptors always are, and ask with
     * their matrix row index k */
    return (A.i / A.mb + k < A.gm / A.mb || A.gm % A.mb == 0) ? A.mb : A.gm % A.mb;
}

/* Width of the tile stored at tile column k. */
PLASMA_HD int plasma_tile_nmain(plasma_desc_t A, int k)
{
    return (A.j / A.nb + k < A.gn / A.nb) ? A.nb : A.gn % A.nb;
}

/* Rows of the view that fall in tile row k. */
PLASMA_HD int plasma_tile_mview(plasma_desc_t A, int k)
{
    if (k < A.mt - 1)
        return A.mb;
    int r = (A.i + A.m) % A.mb;
    return r == 0 ? A.mb : r;
}

/* Columns of the view that fall in tile column k. */
PLASMA_HD int plasma_tile_nview(plasma_desc_t A, int k)
{
    if (k < A.nt - 1)
        return A.nb;
    int r = (A.j + A.n) % A.nb;
    return r == 0 ? A.nb : r;
}

/* reference control/descriptor.c:16-47 (storage is device memory here) */
int plasma_desc_general_create(plasma_enum_t precision, int mb, int nb,
                               int lm, int ln, int i, int j, int m, int n,
                               plasma_desc_t *A);
/* reference control/descriptor.c:85-119 (packed triangle, device memory) */
int plasma_desc_triangular_create(plasma_enum_t precision, plasma_enum_t uplo,
                                  int mb, int nb, int lm, int ln,
                                  int i, int j, int m, int n,
                                  plasma_desc_t *A);
/* reference control/descriptor.c:122-131 */
int plasma_desc_destroy(plasma_desc_t *A);
/* reference control/descriptor.c:134-175 */
int plasma_desc_general_init(plasma_enum_t precision, void *matrix,
                             int mb, int nb, int lm, int ln, int i, int j,
                             int m, int n, plasma_desc_t *A);
/* reference control/descriptor.c:216-264 */
int plasma_desc_triangular_init(plasma_enum_t precision, plasma_enum_t uplo,
                                void *matrix, int mb, int nb, int lm, int ln,
                                int i, int j, int m, int n, plasma_desc_t *A);
/* reference control/descriptor.c:50-82 (band storage, device memory) */
int plasma_desc_general_band_create(plasma_enum_t precision, plasma_enum_t uplo,
                                    int mb, int nb, int lm, int ln,
                                    int i, int j, int m, int n, int kl, int ku,
                                    plasma_desc_t *A);
/* reference control/descriptor.c:178-213 */
int plasma_desc_general_band_init(plasma_enum_t precision, plasma_enum_t uplo,
                                  void *matrix, int mb, int nb, int lm, int ln,
                                  int i, int j, int m, int n, int kl, int ku,
                                  plasma_desc_t *A);
/* reference control/descriptor.c:267-319 */
int plasma_desc_check(plasma_desc_t A);
int plasma_desc_general_check(plasma_desc_t A);
/* reference control/descriptor.c:321-369 */
int plasma_desc_general_band_check(plasma_desc_t A);
/* reference control/descriptor.c:374-397 */
plasma_desc_t plasma_desc_view(plasma_desc_t A, int i, int j, int m, int n);

/* Bytes of storage a descriptor of this shape needs (GPU-build helper). */
size_t plasma_desc_storage_bytes(plasma_desc_t A);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_DESCRIPTOR_H */
