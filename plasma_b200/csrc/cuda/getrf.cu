// getrf.cu -- LU factorization with partial pivoting and its solves, the
// kernels of the LU-based mixed-precision solver (plasma_dsgesv).
//
// The reference's tile LU (compute/pzgetrf.c:37-232) factors each tile
// column as a panel -- pivot search over the whole column below the
// diagonal, row interchange, scaling, rank-1 update (core_blas/
// core_zgetrf.c:20-238) -- then applies the panel's interchanges to the other
// columns (geswp), solves the block row with the unit-lower diagonal tile
// (trsm) and updates the trailing matrix (gemm).  Here:
//   k_getrf_panel   the panel of one tile column in one CTA: the rows of the
//                   panel are strided over 1024 threads, the pivot is found
//                   by a warp-shuffle then shared-memory max reduction (the
//                   first entry of largest magnitude, as LAPACK's idamax),
//                   and each thread applies the rank-1 update to its rows;
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

constexpr int kPanelThreads = 1024;

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

template <typename T>
__global__ void __launch_bounds__(kPanelThreads)
k_getrf_panel(plasma_desc_t A, int k, int *ipiv, plasma_devstat_t *st, int call)
{
    __shared__ T s_val[kPanelThreads / 32];
    __shared__ int s_idx[kPanelThreads / 32];
    __shared__ int s_piv, s_zero;
    if (plasma_failed(st)) return;
    const int r0 = k * A.mb;                       // first row of the panel
    const int M = A.m - r0;                        // panel rows
    const int kb = min(plasma_tile_nview(A, k), M);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;

    for (int j = 0; j < kb; j++) {
        // pivot search down column j from row j
        T bv = T(-1);
        int bi = INT_MAX;
        for (int r = j + tid; r < M; r += blockDim.x)
            max_pick(bv, bi, (T)fabs(*panel_at<T>(A, k, r, j)), r);
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
            bv = lane < nwarps ? s_val[lane] : T(-1);
            bi = lane < nwarps ? s_idx[lane] : INT_MAX;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                max_pick(bv, bi, __shfl_xor_sync(0xffffffffu, bv, o),
                         __shfl_xor_sync(0xffffffffu, bi, o));
            if (lane == 0) {
                // a column of NaNs has no larger entry: keep the diagonal one
                const int p = bi == INT_MAX ? j : bi;
                s_piv = p;
                s_zero = *panel_at<T>(A, k, p, j) == T(0);
                ipiv[r0 + j] = r0 + p + 1;
                if (s_zero)
                    plasma_fail(st, r0 + j + 1, call);
            }
        }
        __syncthreads();
        if (s_zero)
            return;                                   // the whole CTA leaves
        const int p = s_piv;
        if (p != j)
            for (int c = tid; c < kb; c += blockDim.x) {
                T *a = panel_at<T>(A, k, j, c), *b = panel_at<T>(A, k, p, c);
                const T t = *a;
                *a = *b;
                *b = t;
            }
        __syncthreads();
        const T piv = *panel_at<T>(A, k, j, j);
        const bool normal = (T)fabs(piv) >= tiny<T>();
        const T rpiv = T(1) / piv;
        for (int r = j + 1 + tid; r < M; r += blockDim.x) {
            T *lr = panel_at<T>(A, k, r, j);
            const T l = normal ? *lr / piv : *lr * rpiv;
            *lr = l;
            for (int c = j + 1; c < kb; c++)
                *panel_at<T>(A, k, r, c) -= l * *panel_at<T>(A, k, j, c);
        }
        __syncthreads();
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

extern "C" void plasma_cuda_getrf_panel(cudaStream_t s, plasma_devstat_t *st, int call,
                                        plasma_desc_t A, int k, int *ipiv)
{
    PLASMA_COUNT_LAUNCH();
    const double M = A.m - k * A.mb, kb = plasma_tile_nview(A, k);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        k_getrf_panel<double><<<1, kPanelThreads, 0, s>>>(A, k, ipiv, st, call);
    else
        k_getrf_panel<float><<<1, kPanelThreads, 0, s>>>(A, k, ipiv, st, call);
    plasma_prof_end(prof, s, PLASMA_KCLASS_POTRF, M * kb * kb - kb * kb * kb / 3.0,
                    2.0 * M * kb * plasma_element_size(A.precision));
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
