// getrf.cu -- LU factorization with partial pivoting and its solves, the
// kernels of the LU-based mixed-precision solver (plasma_dsgesv).
//
// The reference's tile LU (compute/pzgetrf.c:37-232) factors each tile
// column as a panel -- pivot search over the whole column below the
// diagonal, row interchange, scaling, rank-1 update (core_blas/
// core_zgetrf.c:20-238) -- then applies the panel's interchanges to the other
// columns (geswp), solves the block row with the unit-lower diagonal tile
// (trsm) and updates the trailing matrix (gemm).  Here:
//   k_lu_pivot,     the panel of one tile column, two launches per column:
//   k_lu_update     the pivot (the first entry of largest magnitude, as
//                   LAPACK's idamax) from per-CTA candidates and the row
//                   interchange in one CTA, then scaling, rank-1 update and
//                   the next column's candidates with a thread per panel row;
//   k_laswp         the interchanges of a range of rows applied to a range of
//                   columns, one thread per column (interchanges of one
//                   column are sequential, columns are independent);
//   k_trtri_lu      inverses of the unit-lower and the upper triangle of
//                   diagonal tiles, one CTA per tile, one thread per column;
//   k_lange_inf     ||A||_inf of a general matrix (row sums, atomic max);
//   k_colmax        columnwise max |x| of an n x nrhs matrix.
// The block-row solve, the trailing update and the block steps of the solves
// are GEMMs on views of the tile matrix (cuda/adjoint.cu, k_gemm_view: DMMA
// for FP64, the three-product TF32 split for FP32).
#include "common.cuh"

#include <float.h>
#include <limits.h>

namespace {

template <typename T> __device__ __forceinline__ T tiny();
template <> __device__ __forceinline__ float tiny<float>() { return FLT_MIN; }
template <> __device__ __forceinline__ double tiny<double>() { return DBL_MIN; }

// Element (r, c) of the panel of tile column k: row r counts from the first
// row of tile row k (the view starts at a tile boundary).
template <typename T>
__device__ __forceinline__ T *panel_at(const plasma_desc_t &A, int k, int r, int c)
{
    const int tm = k + r / A.mb;
    T *t = (T *)plasma_tile_addr(A, tm, k);
    return t + (size_t)c * plasma_tile_mmain(A, tm) + (r - (tm - k) * A.mb);
}

// larger |value| wins; on equal values the smaller row index
template <typename T>
__device__ __forceinline__ void max_pick(T &v, int &i, T ov, int oi)
{
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
}

// The panel of tile column k, one column j at a time, in two launches:
//   k_lu_pivot   (one CTA) reduces the per-CTA candidates of column j to the
//                pivot p (first largest magnitude), records ipiv, records
//                info on an exact zero pivot, and swaps rows j and p across
//                the panel's columns;
//   k_lu_update  (a thread per panel row) scales column j below the pivot,
//                applies the rank-1 update to the rest of its sub-block of
//                kIB columns and, in the same pass, leaves each CTA's
//                candidate for the next column (j = -1: candidates only);
//   k_lu_trsm_block  the sub-block's rows of the panel's later columns.
// Rows r of the panel count from the first row of tile row k.
constexpr int kRows = 256;      // panel rows per CTA of k_lu_update
constexpr int kIB = 32;         // columns of a panel sub-block

template <typename T>
__device__ __forceinline__ void block_best(T &bv, int &bi, T *s_val, int *s_idx)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        max_pick(bv, bi, __shfl_xor_sync(0xffffffffu, bv, o),
                 __shfl_xor_sync(0xffffffffu, bi, o));
    if (lane == 0) {
        s_val[warp] = bv;
        s_idx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        bv = lane < nw ? s_val[lane] : T(-1);
        bi = lane < nw ? s_idx[lane] : INT_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            max_pick(bv, bi, __shfl_xor_sync(0xffffffffu, bv, o),
                     __shfl_xor_sync(0xffffffffu, bi, o));
    }
}

template <typename T>
__global__ void __launch_bounds__(kRows)
k_lu_update(plasma_desc_t A, int k, int j, int ce, int next, T *pval, int *pidx,
            const plasma_devstat_t *st)
{
    __shared__ T s_u[kIB];
    __shared__ T s_val[kRows / 32];
    __shared__ int s_idx[kRows / 32];
    if (plasma_failed(st)) return;
    const int M = A.m - k * A.mb;
    const int r = blockIdx.x * kRows + threadIdx.x;
    if (j >= 0) {
        // the pivot row's entries in the rest of the sub-block (ce - j - 1
        // < kIB of them), shared by the CTA
        for (int c = j + 1 + (int)threadIdx.x; c < ce; c += kRows)
            s_u[c - j - 1] = *panel_at<T>(A, k, j, c);
        __syncthreads();
        if (r < M && r > j) {
            const T piv = *panel_at<T>(A, k, j, j);
            T *lr = panel_at<T>(A, k, r, j);
            const T l = (T)fabs(piv) >= tiny<T>() ? *lr / piv : *lr * (T(1) / piv);
            *lr = l;
            for (int c = j + 1; c < ce; c++)
                *panel_at<T>(A, k, r, c) -= l * s_u[c - j - 1];
        }
    }
    if (next < 0) return;                            // no candidates wanted
    T bv = T(-1);
    int bi = INT_MAX;
    if (r < M && r >= next)
        max_pick(bv, bi, (T)fabs(*panel_at<T>(A, k, r, next)), r);
    block_best(bv, bi, s_val, s_idx);
    if (threadIdx.x == 0) {
        pval[blockIdx.x] = bv;
        pidx[blockIdx.x] = bi;
    }
}

// The rows [s0, ce) of the panel right of the sub-block, columns [ce, kb):
// U12 <- inv(L11) U12 with L11 the unit-lower sub-block diagonal, a thread per
// column (forward substitution down ce - s0 <= kIB rows).
template <typename T>
__global__ void __launch_bounds__(kRows)
k_lu_trsm_block(plasma_desc_t A, int k, int s0, int ce, int kb, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int c = ce + blockIdx.x * kRows + threadIdx.x;
    if (c >= kb) return;
    for (int i = s0 + 1; i < ce; i++) {
        T s = *panel_at<T>(A, k, i, c);
        for (int l = s0; l < i; l++)
            s -= *panel_at<T>(A, k, i, l) * *panel_at<T>(A, k, l, c);
        *panel_at<T>(A, k, i, c) = s;
    }
}

template <typename T>
__global__ void __launch_bounds__(kRows)
k_lu_pivot(plasma_desc_t A, int k, int j, int kb, const T *pval, const int *pidx,
           int nparts, int *ipiv, plasma_devstat_t *st, int call)
{
    __shared__ T s_val[kRows / 32];
    __shared__ int s_idx[kRows / 32];
    __shared__ int s_piv, s_zero;
    if (plasma_failed(st)) return;
    T bv = T(-1);
    int bi = INT_MAX;
    for (int q = threadIdx.x; q < nparts; q += kRows)
        max_pick(bv, bi, pval[q], pidx[q]);
    block_best(bv, bi, s_val, s_idx);
    if (threadIdx.x == 0) {
        // a column of NaNs has no larger entry: keep the diagonal one
        const int p = bi == INT_MAX ? j : bi;
        s_piv = p;
        s_zero = *panel_at<T>(A, k, p, j) == T(0);
        ipiv[k * A.mb + j] = k * A.mb + p + 1;
        if (s_zero)
            plasma_fail(st, k * A.mb + j + 1, call);
    }
    __syncthreads();
    const int p = s_piv;
    if (s_zero || p == j) return;
    for (int c = threadIdx.x; c < kb; c += kRows) {
        T *a = panel_at<T>(A, k, j, c), *b = panel_at<T>(A, k, p, c);
        const T t = *a;
        *a = *b;
        *b = t;
    }
}

// Rows j0 .. j1-1 interchanged with rows ipiv[j]-1 (in order), in columns
// [c0, c1) of D.
template <typename T>
__global__ void __launch_bounds__(128)
k_laswp(plasma_desc_t D, const int *ipiv, int j0, int j1, int c0, int c1,
        const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    const int tn = c / D.nb, cc = c - tn * D.nb;
    for (int j = j0; j < j1; j++) {
        const int p = ipiv[j] - 1;
        if (p == j) continue;
        const int tj = j / D.mb, tp = p / D.mb;
        T *a = (T *)plasma_tile_addr(D, tj, tn) + (size_t)cc * plasma_tile_mmain(D, tj) +
               (j - tj * D.mb);
        T *b = (T *)plasma_tile_addr(D, tp, tn) + (size_t)cc * plasma_tile_mmain(D, tp) +
               (p - tp * D.mb);
        const T t = *a;
        *a = *b;
        *b = t;
    }
}

// For the diagonal tiles k in [k0, k0 + gridDim.x): WL_k = inv(unit lower
// part), WU_k = inv(upper part), each nb x nb column-major (ld nb) at
// W + k*nb*nb; only the leading kb x kb block of a ragged tile is written.
// Thread j computes column j of both inverses by substitution.
template <typename T>
__global__ void __launch_bounds__(512)
k_trtri_lu(plasma_desc_t A, int k0, T *WL, T *WU, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int k = k0 + blockIdx.x;
    const int kb = plasma_tile_mview(A, k);
    const int nb = A.mb;
    const T *a = (const T *)plasma_tile_addr(A, k, k);
    const int lda = plasma_tile_mmain(A, k);
    T *wl = WL + (size_t)k * nb * nb, *wu = WU + (size_t)k * nb * nb;
    for (int j = threadIdx.x; j < kb; j += blockDim.x) {
        T *xl = wl + (size_t)j * nb, *xu = wu + (size_t)j * nb;
        // L X = e_j, L unit lower: x_i = 0 (i < j), x_j = 1, then down
        for (int i = 0; i < j; i++) xl[i] = T(0);
        xl[j] = T(1);
        for (int i = j + 1; i < kb; i++) {
            T s = T(0);
            for (int l = j; l < i; l++) s += a[(size_t)l * lda + i] * xl[l];
            xl[i] = -s;
        }
        // U X = e_j: x_i = 0 (i > j), x_j = 1/u_jj, then up
        for (int i = j + 1; i < kb; i++) xu[i] = T(0);
        xu[j] = T(1) / a[(size_t)j * lda + j];
        for (int i = j - 1; i >= 0; i--) {
            T s = T(0);
            for (int l = i + 1; l <= j; l++) s += a[(size_t)l * lda + i] * xu[l];
            xu[i] = -s / a[(size_t)i * lda + i];
        }
    }
}

// max over rows of sum_j |a_ij| into *out (non-negative doubles compare as
// their bit patterns); *out must start at 0.
template <typename T>
__global__ void __launch_bounds__(256)
k_lange_inf(plasma_desc_t A, double *out, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.m) return;
    const int tm = i / A.mb, ii = i - tm * A.mb;
    const int ld = plasma_tile_mmain(A, tm);
    double s = 0.0;
    for (int tn = 0; tn < A.nt; tn++) {
        const T *t = (const T *)plasma_tile_addr(A, tm, tn) + ii;
        const int w = plasma_tile_nview(A, tn);
        for (int c = 0; c < w; c++) s += fabs((double)t[(size_t)c * ld]);
    }
    atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(s));
}

// out[j] = max_i |D(i, j)| (out zeroed by the caller), one CTA per column
template <typename T>
__global__ void __launch_bounds__(256)
k_colmax(plasma_desc_t D, double *out, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int j = blockIdx.x;
    const int tn = j / D.nb, cc = j - tn * D.nb;
    double m = 0.0;
    for (int i = threadIdx.x; i < D.m; i += blockDim.x) {
        const int tm = i / D.mb;
        const T *t = (const T *)plasma_tile_addr(D, tm, tn);
        const double v = fabs((double)t[(size_t)cc * plasma_tile_mmain(D, tm) + (i - tm * D.mb)]);
        m = v > m ? v : m;
    }
    atomicMax((unsigned long long *)&out[j], (unsigned long long)__double_as_longlong(m));
}

}  // namespace

// parts: room for ceil((A.m - k*mb) / 256) candidate pairs (values of the
// precision of A, then ints).
// The panel in sub-blocks of kIB columns (the blocked right-looking order of
// LAPACK's dgetrf applied inside the panel): each column's rank-1 update
// stops at the end of its sub-block; after the sub-block, its rows of the
// panel's remaining columns are solved with the sub-block's unit-lower
// diagonal and the rows below take one GEMM update.  Interchanges always
// swap whole panel rows.
extern "C" void plasma_cuda_getrf_panel(cudaStream_t s, plasma_devstat_t *st, int call,
                                        plasma_desc_t A, int k, int *ipiv, void *parts)
{
    const int M = A.m - k * A.mb;
    const int kb = min(plasma_tile_nview(A, k), M);
    if (kb <= 0) return;
    const int G = (M + kRows - 1) / kRows;
    const size_t es = plasma_element_size(A.precision);
    int *pidx = (int *)((char *)parts + (((size_t)G * es + 15) & ~(size_t)15));
    const bool dp = A.precision == PlasmaRealDouble;
    auto update = [&](int j, int ce, int next) {
        PLASMA_COUNT_LAUNCH();
        if (dp)
            k_lu_update<double><<<G, kRows, 0, s>>>(A, k, j, ce, next, (double *)parts, pidx,
                                                    st);
        else
            k_lu_update<float><<<G, kRows, 0, s>>>(A, k, j, ce, next, (float *)parts, pidx,
                                                   st);
    };
    int prof = plasma_prof_begin(s);
    const int d0 = k * A.mb;                     // first row and column of the panel
    for (int s0 = 0; s0 < kb; s0 += kIB) {
        const int ce = min(kb, s0 + kIB);
        update(-1, ce, s0);                      // candidates of column s0
        for (int j = s0; j < ce; j++) {
            PLASMA_COUNT_LAUNCH();
            if (dp)
                k_lu_pivot<double><<<1, kRows, 0, s>>>(A, k, j, kb, (const double *)parts,
                                                       pidx, G, ipiv, st, call);
            else
                k_lu_pivot<float><<<1, kRows, 0, s>>>(A, k, j, kb, (const float *)parts,
                                                      pidx, G, ipiv, st, call);
            update(j, ce, j + 1 < ce ? j + 1 : -1);
        }
        if (ce < kb) {
            PLASMA_COUNT_LAUNCH();
            const unsigned g = (unsigned)((kb - ce + kRows - 1) / kRows);
            if (dp)
                k_lu_trsm_block<double><<<g, kRows, 0, s>>>(A, k, s0, ce, kb, st);
            else
                k_lu_trsm_block<float><<<g, kRows, 0, s>>>(A, k, s0, ce, kb, st);
            if (ce < M) {
                plasma_view_t a{}, b{}, c{};
                a.D = b.D = c.D = A;
                a.r0 = d0 + ce;  a.c0 = d0 + s0;         // L21
                b.r0 = d0 + s0;  b.c0 = d0 + ce;         // U12
                c.r0 = d0 + ce;  c.c0 = d0 + ce;         // A22
                plasma_cuda_gemm_view(s, st, M - ce, kb - ce, ce - s0, -1.0, a, b, 1.0, c, 0,
                                      0);
            }
        }
    }
    plasma_prof_end(prof, s, PLASMA_KCLASS_POTRF,
                    (double)M * kb * kb - (double)kb * kb * kb / 3.0,
                    2.0 * (double)M * kb * es);
}

extern "C" size_t plasma_cuda_getrf_parts_bytes(plasma_desc_t A)
{
    const size_t G = (size_t)(A.m + kRows - 1) / kRows;
    return ((G * 8 + 15) & ~(size_t)15) + G * sizeof(int) + 64;
}

extern "C" void plasma_cuda_laswp(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                                  const int *ipiv, int j0, int j1, int c0, int c1)
{
    if (c1 <= c0 || j1 <= j0) return;
    PLASMA_COUNT_LAUNCH();
    const unsigned grid = (unsigned)((c1 - c0 + 127) / 128);
    if (D.precision == PlasmaRealDouble)
        k_laswp<double><<<grid, 128, 0, s>>>(D, ipiv, j0, j1, c0, c1, st);
    else
        k_laswp<float><<<grid, 128, 0, s>>>(D, ipiv, j0, j1, c0, c1, st);
}

extern "C" void plasma_cuda_trtri_lu(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                     int k0, int k1, void *WL, void *WU)
{
    if (k1 <= k0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        k_trtri_lu<double><<<k1 - k0, 512, 0, s>>>(A, k0, (double *)WL, (double *)WU, st);
    else
        k_trtri_lu<float><<<k1 - k0, 512, 0, s>>>(A, k0, (float *)WL, (float *)WU, st);
}

extern "C" void plasma_cuda_lange_inf(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                      double *dnorm)
{
    cudaMemsetAsync(dnorm, 0, sizeof(double), s);
    if (A.m == 0 || A.n == 0) return;
    PLASMA_COUNT_LAUNCH();
    const unsigned grid = (unsigned)((A.m + 255) / 256);
    if (A.precision == PlasmaRealDouble)
        k_lange_inf<double><<<grid, 256, 0, s>>>(A, dnorm, st);
    else
        k_lange_inf<float><<<grid, 256, 0, s>>>(A, dnorm, st);
}

extern "C" void plasma_cuda_colmax(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                                   double *out)
{
    if (D.n == 0) return;
    cudaMemsetAsync(out, 0, sizeof(double) * (size_t)D.n, s);
    if (D.m == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (D.precision == PlasmaRealDouble)
        k_colmax<double><<<D.n, 256, 0, s>>>(D, out, st);
    else
        k_colmax<float><<<D.n, 256, 0, s>>>(D, out, st);
}
