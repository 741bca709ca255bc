// layout.cu -- LAPACK column-major <-> tile layout, tile copies, tile
// additions and precision conversions.
//
// Replaces the per-tile lacpy tasks of the reference's layout converters
// (compute/pzge2desc.c:38-55, pztr2desc.c:31-50, pzdesc2ge.c, pzdesc2tr.c,
// and for band storage pzpb2desc.c, pzdesc2pb.c),
// pzlacpy.c, pzgeadd.c, pzlag2c.c:47-85 and pclag2z.c:28-67 with one launch
// per whole-matrix operation: one CTA per tile, threads striding down the
// rows of a column so that global accesses are coalesced.  All kernels are
// HBM-bandwidth bound (one read and one write of every element).
#include "common.cuh"

#include <float.h>
#include <limits.h>

namespace {

constexpr int kThreads = 256;

// Tile (m,n) of the view of A is visited when the uplo filter admits it.
__device__ __forceinline__ bool tile_in(int uplo, int m, int n)
{
    return uplo == PlasmaLower ? n <= m : uplo == PlasmaUpper ? n >= m : true;
}

// Rows [y1,y2) x cols [x1,x2) of tile (m,n) that belong to the view
// (reference compute/pzge2desc.c:42-46).
struct TileBox {
    int y1, y2, x1, x2;
};
__device__ __forceinline__ TileBox tile_box(const plasma_desc_t &A, int m, int n)
{
    TileBox b;
    b.x1 = n == 0 ? A.j % A.nb : 0;
    b.y1 = m == 0 ? A.i % A.mb : 0;
    b.x2 = n == A.nt - 1 ? (A.j + A.n - 1) % A.nb + 1 : A.nb;
    b.y2 = m == A.mt - 1 ? (A.i + A.m - 1) % A.mb + 1 : A.mb;
    return b;
}

template <typename T, bool TO_TILE>
__global__ void __launch_bounds__(kThreads)
k_lapack_tile(plasma_desc_t A, int uplo, T *pA, int lda, int n0,
              const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    int m = blockIdx.x, n = blockIdx.y + n0;
    if (!tile_in(uplo, m, n)) return;
    TileBox b = tile_box(A, m, n);
    T *tile = (T *)plasma_tile_addr(A, m, n);
    int ldt = plasma_tile_mmain(A, m);
    T *f77 = pA + (size_t)A.nb * lda * n + (size_t)A.mb * m;
    int rows = b.y2 - b.y1;
    int total = rows * (b.x2 - b.x1);
    for (int e = threadIdx.x; e < total; e += kThreads) {
        int y = b.y1 + e % rows;
        int x = b.x1 + e / rows;
        if (TO_TILE)
            tile[(size_t)x * ldt + y] = f77[(size_t)x * lda + y];
        else
            f77[(size_t)x * lda + y] = tile[(size_t)x * ldt + y];
    }
}

// B(m,n) <- A(m,n) with optional precision conversion and the dlag2s
// overflow test (info = 1 when |a| > FLT_MAX; NaN passes, as in LAPACK).
template <typename TA, typename TB, bool CHECK>
__global__ void __launch_bounds__(kThreads)
k_tile_copy(plasma_desc_t A, plasma_desc_t B, int uplo, int n0,
            plasma_devstat_t *st, int call)
{
    if (plasma_failed(st)) return;
    int m = blockIdx.x, n = blockIdx.y + n0;
    if (!tile_in(uplo, m, n)) return;
    // source and destination may have different (padded) shapes
    int rows = min(plasma_tile_mview(A, m), plasma_tile_mview(B, m));
    int cols = min(plasma_tile_nview(A, n), plasma_tile_nview(B, n));
    const TA *a = (const TA *)plasma_tile_addr(A, m, n);
    TB *b = (TB *)plasma_tile_addr(B, m, n);
    int lda = plasma_tile_mmain(A, m);
    int ldb = plasma_tile_mmain(B, m);
    bool overflow = false;
    for (int e = threadIdx.x; e < rows * cols; e += kThreads) {
        int y = e % rows, x = e / rows;
        TA v = a[(size_t)x * lda + y];
        if (CHECK && (v > (TA)FLT_MAX || v < -(TA)FLT_MAX))
            overflow = true;
        b[(size_t)x * ldb + y] = (TB)v;
    }
    if (CHECK && __syncthreads_or(overflow) && threadIdx.x == 0)
        plasma_fail(st, 1, call);
}

// Lower tile (m,n) of an upload in flight, in one pass over the staged
// column-major copy: the FP64 tile of A and its FP32 conversion into As
// (dlag2s overflow test into st).  The kernel never returns early on the
// device status: the FP64 tiles are needed whatever the FP32 factorization
// reports (later attempts and the FP64 fallback read them).  Warps take
// columns, lanes consecutive rows.
__global__ void __launch_bounds__(kThreads)
k_upload_tile(plasma_desc_t A, plasma_desc_t As, const double *src, int ld, int n0,
              plasma_devstat_t *st, int call)
{
    const int m = blockIdx.x, n = blockIdx.y + n0;
    if (n > m) return;
    const TileBox b = tile_box(A, m, n);
    double *t = (double *)plasma_tile_addr(A, m, n);
    float *ts = (float *)plasma_tile_addr(As, m, n);
    const int ldt = plasma_tile_mmain(A, m), lds = plasma_tile_mmain(As, m);
    const double *f = src + (size_t)A.nb * ld * n + (size_t)A.mb * m;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bool overflow = false;
    for (int x = b.x1 + warp; x < b.x2; x += kThreads / 32) {
        const double *fc = f + (size_t)x * ld;
        double *tc = t + (size_t)x * ldt;
        float *sc = ts + (size_t)x * lds;
#pragma unroll 4
        for (int y = b.y1 + lane; y < b.y2; y += 32) {
            const double v = fc[y];
            tc[y] = v;
            if (v > (double)FLT_MAX || v < -(double)FLT_MAX) overflow = true;
            sc[y] = (float)v;
        }
    }
    if (__syncthreads_or(overflow) && threadIdx.x == 0)
        plasma_fail(st, 1, call);
}

// info of dtrtri on the factor held in A: the smallest i with A(i,i) == 0
// (one CTA; the diagonal has n elements)
template <typename T>
__global__ void __launch_bounds__(1024)
k_diag_zero_info(plasma_desc_t A, plasma_devstat_t *st, int call)
{
    __shared__ int first;
    if (threadIdx.x == 0) first = INT_MAX;
    __syncthreads();
    for (int i = threadIdx.x; i < A.m; i += blockDim.x) {
        const int m = i / A.mb, r = i - m * A.mb;
        const T *t = (const T *)plasma_tile_addr(A, m, m);
        if (t[(size_t)r * plasma_tile_mmain(A, m) + r] == T(0)) atomicMin(&first, i);
    }
    __syncthreads();
    if (threadIdx.x == 0 && first != INT_MAX) plasma_fail(st, first + 1, call);
}

// A <- the uplo triangle of B, tile by tile (diagonal tiles: only the uplo
// part, the rest of A stays as it is); A and B have the same tiling
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_copy_uplo(plasma_desc_t B, plasma_desc_t A, int uplo, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int m = blockIdx.x, n = blockIdx.y;
    if (!tile_in(uplo, m, n)) return;
    const T *b = (const T *)plasma_tile_addr(B, m, n);
    T *a = (T *)plasma_tile_addr(A, m, n);
    const int ldb = plasma_tile_mmain(B, m), lda = plasma_tile_mmain(A, m);
    const int rows = plasma_tile_mview(A, m), cols = plasma_tile_nview(A, n);
    const bool diag = m == n, lower = uplo == PlasmaLower;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int x = warp; x < cols; x += kThreads / 32)
        for (int y = lane; y < rows; y += 32)
            if (!diag || (lower ? y >= x : y <= x))
                a[(size_t)x * lda + y] = b[(size_t)x * ldb + y];
}

// B(m,n) <- A(n,m)^T for the lower tiles of B (m >= n) from the upper tiles
// of A (same symmetric matrix in the other triangle), FP64 -> FP32 with the
// overflow test; 32 x 32 blocks transposed through shared memory so that
// both the read and the write run along tile columns.
__global__ void __launch_bounds__(kThreads)
k_tile_copy_t(plasma_desc_t A, plasma_desc_t B, plasma_devstat_t *st, int call)
{
    __shared__ float blk[32][33];
    const int m = blockIdx.x, n = blockIdx.y;
    // one answer for the whole block: the loop below holds barriers
    if (m < n || __syncthreads_or(plasma_failed(st))) return;
    const double *a = (const double *)plasma_tile_addr(A, n, m);
    float *b = (float *)plasma_tile_addr(B, m, n);
    const int lda = plasma_tile_mmain(A, n), ldb = plasma_tile_mmain(B, m);
    // B(m,n) element (i, j) = A(n,m) element (j, i)
    const int rows = min(plasma_tile_mview(B, m), plasma_tile_nview(A, m));
    const int cols = min(plasma_tile_nview(B, n), plasma_tile_mview(A, n));
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    bool overflow = false;
    for (int i0 = 0; i0 < rows; i0 += 32)
        for (int j0 = 0; j0 < cols; j0 += 32) {
            __syncthreads();
            // read A(n,m)(j0 + tx, i0 + q): along A's columns
            for (int q = ty; q < 32; q += kThreads / 32) {
                const int j = j0 + tx, i = i0 + q;
                float v = 0.f;
                if (j < cols && i < rows && (m != n || i >= j)) {
                    const double x = a[(size_t)i * lda + j];
                    if (x > (double)FLT_MAX || x < -(double)FLT_MAX) overflow = true;
                    v = (float)x;
                }
                blk[q][tx] = v;                       // blk[i - i0][j - j0]
            }
            __syncthreads();
            // write B(m,n)(i0 + tx, j0 + q): along B's columns
            for (int q = ty; q < 32; q += kThreads / 32) {
                const int i = i0 + tx, j = j0 + q;
                if (i < rows && j < cols && (m != n || i >= j))
                    b[(size_t)j * ldb + i] = blk[tx][q];
            }
        }
    if (__syncthreads_or(overflow) && threadIdx.x == 0)
        plasma_fail(st, 1, call);
}

// The lower tiles of B (m >= n) <-> the upper triangle of the column-major
// array pA, transposed: tile (m,n) element (i,j) is pA(r, c) with
// r = n*nb + j <= c = m*nb + i, i.e. B holds U^T = L when pA holds the
// upper triangle U of a symmetric matrix.  Used for upper storage, whose
// factor is the transpose of the lower one, so that the tensor-core tile
// kernels (written for lower tiles) factor it.  32 x 32 blocks go through
// shared memory so that both sides are read and written along their
// columns.  The strictly upper part of a diagonal tile (the strictly lower
// part of pA) is zero on the way in and not written on the way out.
template <typename T, bool TO_TILE>
__global__ void __launch_bounds__(kThreads)
k_lapack_tile_t(plasma_desc_t B, T *pA, int lda, const plasma_devstat_t *st)
{
    __shared__ T blk[32][33];
    const int m = blockIdx.x, n = blockIdx.y;
    if (m < n || __syncthreads_or(plasma_failed(st))) return;
    T *tile = (T *)plasma_tile_addr(B, m, n);
    const int ldt = plasma_tile_mmain(B, m);
    const int rows = plasma_tile_mview(B, m), cols = plasma_tile_nview(B, n);
    // pA(n*nb + j, m*nb + i) = f[j + i*lda]
    T *f = pA + (size_t)B.mb * m * lda + (size_t)B.nb * n;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const bool diag = m == n;
    for (int i0 = 0; i0 < rows; i0 += 32)
        for (int j0 = 0; j0 < cols; j0 += 32) {
            __syncthreads();
            if (TO_TILE) {
                // read along pA's columns: j = j0 + tx contiguous
                for (int q = ty; q < 32; q += kThreads / 32) {
                    const int j = j0 + tx, i = i0 + q;
                    T v = T(0);
                    if (j < cols && i < rows && (!diag || i >= j))
                        v = f[(size_t)i * lda + j];
                    blk[q][tx] = v;                    // blk[i - i0][j - j0]
                }
                __syncthreads();
                for (int q = ty; q < 32; q += kThreads / 32) {
                    const int i = i0 + tx, j = j0 + q;
                    if (i < rows && j < cols)
                        tile[(size_t)j * ldt + i] = blk[tx][q];
                }
            } else {
                // read along the tile's columns: i = i0 + tx contiguous
                for (int q = ty; q < 32; q += kThreads / 32) {
                    const int i = i0 + tx, j = j0 + q;
                    blk[q][tx] = (i < rows && j < cols) ? tile[(size_t)j * ldt + i] : T(0);
                }
                __syncthreads();                       // blk[j - j0][i - i0]
                for (int q = ty; q < 32; q += kThreads / 32) {
                    const int j = j0 + tx, i = i0 + q;
                    if (j < cols && i < rows && (!diag || i >= j))
                        f[(size_t)i * lda + j] = blk[tx][q];
                }
            }
        }
}

// X(m,n) += R(m,n)  (reference compute/pzgeadd.c:28-73 with alpha = beta = 1)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_tile_add(plasma_desc_t R, plasma_desc_t X, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    int m = blockIdx.x, n = blockIdx.y;
    int rows = plasma_tile_mview(X, m);
    int cols = plasma_tile_nview(X, n);
    const T *r = (const T *)plasma_tile_addr(R, m, n);
    T *x = (T *)plasma_tile_addr(X, m, n);
    int ldr = plasma_tile_mmain(R, m);
    int ldx = plasma_tile_mmain(X, m);
    for (int e = threadIdx.x; e < rows * cols; e += kThreads) {
        int y = e % rows, c = e / rows;
        x[(size_t)c * ldx + y] += r[(size_t)c * ldr + y];
    }
}

// A(i,i) = v for i in [i0, i1)
template <typename T>
__global__ void k_set_diag(plasma_desc_t A, int i0, int i1, T v)
{
    int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= i1) return;
    int m = i / A.mb, r = i % A.mb;
    T *t = (T *)plasma_tile_addr(A, m, m);
    t[(size_t)r * plasma_tile_mmain(A, m) + r] = v;
}

// LAPACK band storage <-> band tile descriptor (the reference's
// compute/pzpb2desc.c:31-61 and pzdesc2pb.c).  Element (i,j) of the band
// (view coordinates) sits at pAB[off + i - j + j*ldab], off = ku for upper
// and 0 for lower storage.  One CTA per stored tile: blockIdx.x walks the
// kut+klt-1 tiles of band column blockIdx.y.  On the way in every element of
// the stored tile is written (zero outside the band and below the matrix),
// so the tile kernels never read stale values; on the way out only band
// elements are written.
template <typename T, bool TO_TILE>
__global__ void __launch_bounds__(kThreads)
k_band_tile(plasma_desc_t A, T *pAB, int ldab, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int n = blockIdx.y;
    const int m = n - (A.kut - 1) + (int)blockIdx.x;
    if (m < 0 || m >= A.mt) return;
    const bool lower = A.uplo == PlasmaLower;
    const int off = lower ? 0 : A.ku;
    const int rows = plasma_tile_mview(A, m);
    const int cols = plasma_tile_nview(A, n);
    T *tile = (T *)plasma_tile_addr(A, m, n);
    const int ldt = plasma_tile_mmain(A, m);
    const int h = TO_TILE ? A.mb : rows;     // stored rows visited
    const int d0 = m * A.mb - n * A.nb;      // i - j at the tile's corner
    for (int e = threadIdx.x; e < h * cols; e += kThreads) {
        const int r = e % h, c = e / h;
        const int d = d0 + r - c;
        const bool in = r < rows && (lower ? (d >= 0 && d <= A.kl) : (d <= 0 && d >= -A.ku));
        const size_t ab = (size_t)(n * A.nb + c) * ldab + (off + d);
        if (TO_TILE)
            tile[(size_t)c * ldt + r] = in ? pAB[ab] : T(0);
        else if (in)
            pAB[ab] = tile[(size_t)c * ldt + r];
    }
}

dim3 tile_grid(const plasma_desc_t &A)
{
    return dim3((unsigned)A.mt, (unsigned)A.nt);
}

}  // namespace

extern "C" void plasma_cuda_lapack_to_tile(cudaStream_t s, plasma_devstat_t *st,
                                           plasma_desc_t A, plasma_enum_t uplo,
                                           const void *pA, int lda)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_lapack_tile<double, true><<<tile_grid(A), kThreads, 0, s>>>(
            A, uplo, (double *)pA, lda, 0, st);
    else
        k_lapack_tile<float, true><<<tile_grid(A), kThreads, 0, s>>>(
            A, uplo, (float *)pA, lda, 0, st);
}

extern "C" void plasma_cuda_tile_to_lapack(cudaStream_t s, plasma_devstat_t *st,
                                           plasma_desc_t A, plasma_enum_t uplo,
                                           void *pA, int lda)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_lapack_tile<double, false><<<tile_grid(A), kThreads, 0, s>>>(
            A, uplo, (double *)pA, lda, 0, st);
    else
        k_lapack_tile<float, false><<<tile_grid(A), kThreads, 0, s>>>(
            A, uplo, (float *)pA, lda, 0, st);
}

// The upper triangle of the column-major pA <-> the lower tiles of B,
// transposed (k_lapack_tile_t); B is a lower (packed or general) descriptor
// of square tiles with B.i = B.j = 0.
extern "C" void plasma_cuda_lapack_to_tile_t(cudaStream_t s, plasma_devstat_t *st,
                                             plasma_desc_t B, const void *pA, int lda)
{
    if (B.mt == 0 || B.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (B.precision == PlasmaRealDouble)
        k_lapack_tile_t<double, true><<<tile_grid(B), kThreads, 0, s>>>(
            B, (double *)pA, lda, st);
    else
        k_lapack_tile_t<float, true><<<tile_grid(B), kThreads, 0, s>>>(
            B, (float *)pA, lda, st);
}

extern "C" void plasma_cuda_tile_to_lapack_t(cudaStream_t s, plasma_devstat_t *st,
                                             plasma_desc_t B, void *pA, int lda)
{
    if (B.mt == 0 || B.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (B.precision == PlasmaRealDouble)
        k_lapack_tile_t<double, false><<<tile_grid(B), kThreads, 0, s>>>(
            B, (double *)pA, lda, st);
    else
        k_lapack_tile_t<float, false><<<tile_grid(B), kThreads, 0, s>>>(
            B, (float *)pA, lda, st);
}

// Band descriptors of lower or upper storage (A.uplo); the caller checks// Band descriptors of lower or upper storage (A.uplo); the caller checks
// ldab >= kl+1 (lower) or ku+1 (upper).
extern "C" void plasma_cuda_band_to_tile(cudaStream_t s, plasma_devstat_t *st,
                                         plasma_desc_t A, const void *pAB, int ldab)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)(A.kut + A.klt - 1), (unsigned)A.nt);
    if (A.precision == PlasmaRealDouble)
        k_band_tile<double, true><<<grid, kThreads, 0, s>>>(A, (double *)pAB, ldab, st);
    else
        k_band_tile<float, true><<<grid, kThreads, 0, s>>>(A, (float *)pAB, ldab, st);
}

extern "C" void plasma_cuda_tile_to_band(cudaStream_t s, plasma_devstat_t *st,
                                         plasma_desc_t A, void *pAB, int ldab)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)(A.kut + A.klt - 1), (unsigned)A.nt);
    if (A.precision == PlasmaRealDouble)
        k_band_tile<double, false><<<grid, kThreads, 0, s>>>(A, (double *)pAB, ldab, st);
    else
        k_band_tile<float, false><<<grid, kThreads, 0, s>>>(A, (float *)pAB, ldab, st);
}

extern "C" void plasma_cuda_lacpy(cudaStream_t s, plasma_devstat_t *st,
                                  plasma_desc_t A, plasma_desc_t B)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_tile_copy<double, double, false><<<tile_grid(A), kThreads, 0, s>>>(
            A, B, PlasmaGeneral, 0, st, 0);
    else
        k_tile_copy<float, float, false><<<tile_grid(A), kThreads, 0, s>>>(
            A, B, PlasmaGeneral, 0, st, 0);
}

// As (lower tiles) <- A held in upper storage: the conversion of dsposv
// when its FP32 factor is kept in lower storage for an upper-stored A.
extern "C" void plasma_cuda_lag2s_upper_to_lower(cudaStream_t s, plasma_devstat_t *st,
                                                 int call, plasma_desc_t A,
                                                 plasma_desc_t As)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    k_tile_copy_t<<<tile_grid(A), kThreads, 0, s>>>(A, As, st, call);
}

extern "C" void plasma_cuda_lag2s(cudaStream_t s, plasma_devstat_t *st, int call,
                                  plasma_desc_t A, plasma_desc_t As,
                                  plasma_enum_t uplo)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    k_tile_copy<double, float, true><<<tile_grid(A), kThreads, 0, s>>>(
        A, As, uplo, 0, st, call);
}

// Tile columns [n0, n1) only: the FP64 tiles of A from a column-major copy
// (src, ld: the whole matrix) and their FP32 conversion into As, lower
// tiles -- the per-group conversion of an upload that runs alongside the
// factorization of the groups before it.
extern "C" void plasma_cuda_upload_cols(cudaStream_t s, plasma_devstat_t *st, int call,
                                        plasma_desc_t A, plasma_desc_t As, const double *src,
                                        int ld, int n0, int n1)
{
    if (n1 <= n0 || A.mt == 0) return;
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)A.mt, (unsigned)(n1 - n0));
    k_upload_tile<<<grid, kThreads, 0, s>>>(A, As, src, ld, n0, st, call);
}

extern "C" void plasma_cuda_diag_zero_info(cudaStream_t s, plasma_devstat_t *st, int call,
                                           plasma_desc_t A)
{
    if (A.m == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_diag_zero_info<double><<<1, 1024, 0, s>>>(A, st, call);
    else
        k_diag_zero_info<float><<<1, 1024, 0, s>>>(A, st, call);
}

extern "C" void plasma_cuda_copy_uplo(cudaStream_t s, plasma_devstat_t *st, plasma_enum_t uplo,
                                      plasma_desc_t B, plasma_desc_t A)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_copy_uplo<double><<<tile_grid(A), kThreads, 0, s>>>(B, A, uplo, st);
    else
        k_copy_uplo<float><<<tile_grid(A), kThreads, 0, s>>>(B, A, uplo, st);
}

extern "C" void plasma_cuda_slag2d(cudaStream_t s, plasma_devstat_t *st,
                                   plasma_desc_t As, plasma_desc_t A)
{
    if (A.mt == 0 || A.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    k_tile_copy<float, double, false><<<tile_grid(As), kThreads, 0, s>>>(
        As, A, PlasmaGeneral, 0, st, 0);
}

extern "C" void plasma_cuda_geadd(cudaStream_t s, plasma_devstat_t *st,
                                  plasma_desc_t R, plasma_desc_t X)
{
    if (X.mt == 0 || X.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (X.precision == PlasmaRealDouble)
        k_tile_add<double><<<tile_grid(X), kThreads, 0, s>>>(R, X, st);
    else
        k_tile_add<float><<<tile_grid(X), kThreads, 0, s>>>(R, X, st);
}

extern "C" void plasma_cuda_set_diag(cudaStream_t s, plasma_desc_t A, int i0,
                                     int i1, double value)
{
    if (i1 <= i0) return;
    PLASMA_COUNT_LAUNCH();
    int n = i1 - i0;
    if (A.precision == PlasmaRealDouble)
        k_set_diag<double><<<(n + 255) / 256, 256, 0, s>>>(A, i0, i1, value);
    else
        k_set_diag<float><<<(n + 255) / 256, 256, 0, s>>>(A, i0, i1, (float)value);
}
