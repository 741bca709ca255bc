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
//   k_lu_panel_cl   the whole panel in one launch when it is at most 64
//                   columns wide and fits a cluster's shared memory;
//   k_laswp_rows    the interchanges of up to 64 rows applied to a range of
//                   columns as one permutation, a warp per column;
//   k_laswp_vec     all interchanges on one column (the solves' right-hand
//                   side), in shared memory;
//   k_trtri_lu      inverses of the unit-lower and the upper triangle of
//                   diagonal tiles, one CTA per tile, one thread per column
//                   (k_trtri_lu64 for 64-wide tiles: FP64 in shared memory,
//                   products on DMMA);
//   k_gemv_part     partial row sums of A x or |A| over ranges of tile
//   k_gemv_finish   columns, then their sum (the residual b - A x) or the
//                   largest one (||A||_inf);
//   k_colmax        columnwise max |x| of an n x nrhs matrix.
// The block-row solve, the trailing update and the block steps of the solves
// are GEMMs on views of the tile matrix (cuda/adjoint.cu, k_gemm_view: DMMA
// for FP64, the three-product TF32 split for FP32).
#include "common.cuh"
#include "inv64.cuh"
#include "mma.cuh"

#include <float.h>
#include <limits.h>
#include <stdlib.h>

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

// The interchanges of the rows [j0, j0 + nj), nj <= 64, in columns
// [c0, c1).  The swaps are the same for every column, so one thread first
// composes them into a permutation of the rows involved -- the block rows
// j0 .. j0+nj-1 and every distinct row below the block that they name, at
// most 128 positions -- and then every column is a gather: a warp per
// column, its lanes over the positions, all reads before the writes.
constexpr int LW_WARPS = 8, LW_COLS_PER_WARP = 4;
constexpr int LW_COLS = LW_WARPS * LW_COLS_PER_WARP;

template <typename T>
__global__ void __launch_bounds__(32 * LW_WARPS)
k_laswp_rows(plasma_desc_t D, const int *ipiv, int j0, int nj, int c0, int c1, int skip0,
             int skip1, const plasma_devstat_t *st)
{
    __shared__ int tgt[64], slot[64], src[128], row[128], pos_of_slot[64];
    __shared__ int npos;
    if (plasma_failed(st)) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < nj) tgt[tid] = ipiv[j0 + tid] - 1;
    __syncthreads();
    // a row below the block gets the slot of the first swap that names it
    if (tid < nj) {
        const int t = tgt[tid];
        int q = -1;
        if (t >= j0 + nj)
            for (q = 0; tgt[q] != t; q++) {}
        slot[tid] = q;
    }
    __syncthreads();
    if (tid == 0) {
        // positions: nj block rows, then the distinct rows below
        int np = nj;
        for (int r = 0; r < nj; r++) {
            row[r] = j0 + r;
            src[r] = r;
        }
        for (int q = 0; q < nj; q++) {
            if (slot[q] == q) {
                pos_of_slot[q] = np;
                row[np] = tgt[q];
                src[np] = np;
                np++;
            }
        }
        for (int j = 0; j < nj; j++) {
            const int t = tgt[j];
            if (t == j0 + j) continue;
            const int pt = t < j0 + nj ? t - j0 : pos_of_slot[slot[j]];
            const int x = src[j];
            src[j] = src[pt];
            src[pt] = x;
        }
        npos = np;
    }
    __syncthreads();
    const int np = npos;
    for (int q = 0; q < LW_COLS_PER_WARP; q++) {
        int c = c0 + blockIdx.x * LW_COLS + warp * LW_COLS_PER_WARP + q;
        if (c >= skip0) c += skip1 - skip0;           // columns [skip0, skip1) are left out
        if (c >= c1) break;
        const int tn = c / D.nb, cc = c - tn * D.nb;
        auto at = [&](int r) -> T * {
            const int tm = r / D.mb;
            return (T *)plasma_tile_addr(D, tm, tn) + (size_t)cc * plasma_tile_mmain(D, tm) +
                   (r - tm * D.mb);
        };
        T v[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const int p = lane + 32 * h;
            if (p < np) v[h] = *at(row[src[p]]);
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const int p = lane + 32 * h;
            if (p < np) *at(row[p]) = v[h];
        }
        __syncwarp();
    }
}

// All interchanges of ipiv[0 .. n) on one column of D, in shared memory:
// one thread walks the swaps (they are sequential), the loads and stores
// around it are spread over the CTA.
template <typename T>
__global__ void __launch_bounds__(256)
k_laswp_vec(plasma_desc_t D, int col, const int *ipiv, int n, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char lv_raw[];
    T *v = reinterpret_cast<T *>(lv_raw);
    int *pv = reinterpret_cast<int *>(v + n);
    if (plasma_failed(st)) return;
    const int tn = col / D.nb, cc = col - tn * D.nb;
    auto at = [&](int r) -> T * {
        const int tm = r / D.mb;
        return (T *)plasma_tile_addr(D, tm, tn) + (size_t)cc * plasma_tile_mmain(D, tm) +
               (r - tm * D.mb);
    };
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        v[r] = *at(r);
        pv[r] = ipiv[r] - 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < n; j++) {
            const int p = pv[j];
            const T x = v[j];
            v[j] = v[p];
            v[p] = x;
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) *at(r) = v[r];
}

// The interchanges ipiv[0 .. n) composed into one permutation, once per
// factorization: perm[i] = the row whose entry ends at row i (one thread
// walks the swaps in shared memory).
__global__ void __launch_bounds__(256)
k_ipiv_perm(const int *ipiv, int n, int *perm, const plasma_devstat_t *st)
{
    extern __shared__ int ip_raw[];
    int *idx = ip_raw, *pv = ip_raw + n;
    if (plasma_failed(st)) return;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        idx[r] = r;
        pv[r] = ipiv[r] - 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < n; j++) {
            const int p = pv[j], x = idx[j];
            idx[j] = idx[p];
            idx[p] = x;
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) perm[r] = idx[r];
}

// column col of D (n rows) <- its rows in the order perm
template <typename T>
__global__ void __launch_bounds__(1024)
k_permute_vec(plasma_desc_t D, int col, const int *perm, int n, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char pm_raw[];
    T *v = reinterpret_cast<T *>(pm_raw);
    if (plasma_failed(st)) return;
    const int tn = col / D.nb, cc = col - tn * D.nb;
    auto at = [&](int r) -> T * {
        const int tm = r / D.mb;
        return (T *)plasma_tile_addr(D, tm, tn) + (size_t)cc * plasma_tile_mmain(D, tm) +
               (r - tm * D.mb);
    };
    for (int r = threadIdx.x; r < n; r += blockDim.x) v[r] = *at(r);
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) *at(r) = v[perm[r]];
}

// 64-wide tiles: CTA 2q inverts the unit-lower part of diagonal tile
// k0 + q, CTA 2q+1 its upper part (through U^T, lower), both in FP64 in
// shared memory (inv_lower64); a ragged tile is padded with the identity.
constexpr int LU_INV_SMEM = (2 * 64 * 65 + 64 * 33) * 8;

template <typename T>
__global__ void __launch_bounds__(256)
k_trtri_lu64(plasma_desc_t A, int k0, T *WL, T *WU, const plasma_devstat_t *st)
{
    extern __shared__ double inv_smem[];
    double (*Ls)[65] = reinterpret_cast<double (*)[65]>(inv_smem);
    double (*Iv)[65] = Ls + 64;
    double (*Tm)[33] = reinterpret_cast<double (*)[33]>(Iv + 64);
    if (plasma_failed(st)) return;
    const int k = k0 + blockIdx.x / 2;
    const bool up = (blockIdx.x & 1) != 0;
    const T *t = (const T *)plasma_tile_addr(A, k, k);
    const int ld = plasma_tile_mmain(A, k);
    const int kb = min(plasma_tile_mview(A, k), plasma_tile_nview(A, k));
    for (int e = threadIdx.x; e < 64 * 64; e += 256) {
        const int i = e % 64, c = e / 64;
        double v;
        if (i >= kb || c >= kb) v = i == c ? 1.0 : 0.0;
        else if (!up) v = i > c ? (double)t[(size_t)c * ld + i] : (i == c ? 1.0 : 0.0);
        else v = i >= c ? (double)t[(size_t)i * ld + c] : 0.0;     // U^T
        Ls[i][c] = v;
        Iv[i][c] = 0.0;
    }
    __syncthreads();
    inv_lower64(Ls, Iv, Tm, !up);
    T *w = (up ? WU : WL) + (size_t)k * A.mb * A.mb;
    for (int e = threadIdx.x; e < 64 * 64; e += 256) {
        const int i = e % 64, c = e / 64;
        if (i < kb && c < kb) w[(size_t)c * A.mb + i] = (T)(up ? Iv[c][i] : Iv[i][c]);
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

// The trailing update of step k for 64 x 64 FP32 tiles,
//     A(m, n) -= A(m, k) A(k, n),   m, n > k,
// on the tensor cores (mma.sync, the three-product TF32 split, FP32
// accuracy).  A CTA owns a 128 x 128 block of C (two tile rows, two tile
// columns) and the whole K = 64: L's two tiles and U's two tiles are copied
// in by 16-byte cp.async (the tiles are contiguous, column-major), L as
// As[k][i] and U as Bs[j][k] (both padded for conflict-free fragment
// loads); eight warps of 64 x 32, then C -= the product in place.
constexpr int LG_THREADS = 256;
constexpr int LG_LDA = 128 + 8, LG_LDB = 64 + 4;
constexpr int LG_SMEM = (64 * LG_LDA + 128 * LG_LDB) * 4;

// acc (a warp's 64 x 32 block at rows wm, columns wn) = As^T-view x Bs over
// K = 64: As[k][i] (rows i), Bs[j][k] (columns j)
__device__ __forceinline__ void lg_product(const float *As, const float *Bs, int wm, int wn,
                                           int g, int t, float (&acc)[4][4][4])
{
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;
#pragma unroll 2
    for (int k8 = 0; k8 < 64; k8 += 8) {
        float bf[4][2];
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
            bf[ni][0] = Bs[(wn + ni * 8 + g) * LG_LDB + k8 + t];
            bf[ni][1] = Bs[(wn + ni * 8 + g) * LG_LDB + k8 + t + 4];
        }
#pragma unroll
        for (int mi = 0; mi < 4; mi++) {
            float af[4];
            af[0] = As[(k8 + t) * LG_LDA + wm + mi * 16 + g];
            af[1] = As[(k8 + t) * LG_LDA + wm + mi * 16 + g + 8];
            af[2] = As[(k8 + t + 4) * LG_LDA + wm + mi * 16 + g];
            af[3] = As[(k8 + t + 4) * LG_LDA + wm + mi * 16 + g + 8];
#pragma unroll
            for (int ni = 0; ni < 4; ni++) mma8<3>(acc[mi][ni], af, bf[ni]);
        }
    }
}

// 64 x 64 column-major tile (ld, rows x cols valid, zero elsewhere) into
// shared memory: as rows (dst[c*ldd + i]) or, transposed, as columns
// (dst[j*ldd + k] = t(k, j), k the row)
__device__ __forceinline__ void lg_stage(float *dst, int ldd, const float *src, int ld,
                                         int rows, int cols, int tid, int nthreads)
{
    for (int e = tid; e < 64 * 16; e += nthreads) {
        const int c = e / 16, q = e % 16;              // column c, rows 4q .. 4q+3
        float *d = &dst[c * ldd + 4 * q];
        if (src != nullptr && c < cols && 4 * q + 3 < rows && (ld & 3) == 0) {
            cp_async_16(d, src + (size_t)c * ld + 4 * q, true);
        } else {
            for (int r = 0; r < 4; r++)
                d[r] = (src != nullptr && c < cols && 4 * q + r < rows)
                           ? src[(size_t)c * ld + 4 * q + r] : 0.f;
        }
    }
}

__global__ void __launch_bounds__(LG_THREADS, 2)
k_lu_gemm(plasma_desc_t A, int k, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) float lg_raw[];
    float *As = lg_raw;                        // [64][LG_LDA]  L(m..m+1, k)
    float *Bs = lg_raw + 64 * LG_LDA;          // [128][LG_LDB] U(k, n..n+1), [j][k]
    if (plasma_failed(st)) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = k + 1 + 2 * blockIdx.y, n0 = k + 1 + 2 * blockIdx.x;
    const int kb = plasma_tile_nview(A, k);
    // operand tiles (a missing second tile, or a ragged one, reads as zero)
    for (int h = 0; h < 2; h++) {
        const int m = m0 + h;
        const bool mv = m < A.mt;
        lg_stage(As + 64 * h, LG_LDA, mv ? (const float *)plasma_tile_addr(A, m, k) : nullptr,
                 mv ? plasma_tile_mmain(A, m) : 0, mv ? plasma_tile_mview(A, m) : 0, kb, tid,
                 LG_THREADS);
        const int n = n0 + h;
        const bool nv = n < A.nt;
        lg_stage(Bs + 64 * h * LG_LDB, LG_LDB,
                 nv ? (const float *)plasma_tile_addr(A, k, n) : nullptr,
                 plasma_tile_mmain(A, k), kb, nv ? plasma_tile_nview(A, n) : 0, tid, LG_THREADS);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
    float acc[4][4][4];
    lg_product(As, Bs, wm, wn, g, t, acc);
    // C -= acc, tile by tile (rows of a fragment are 8 apart, columns 2t, 2t+1)
#pragma unroll
    for (int mi = 0; mi < 4; mi++) {
        const int rr = wm + mi * 16;                   // 16 rows of one C tile
        const int m = m0 + rr / 64;
        if (m >= A.mt) continue;
        const int rows = plasma_tile_mview(A, m), ld = plasma_tile_mmain(A, m);
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
            const int cc = wn + ni * 8;
            const int n = n0 + cc / 64;
            if (n >= A.nt) continue;
            const int cols = plasma_tile_nview(A, n);
            float *c = (float *)plasma_tile_addr(A, m, n);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = rr % 64 + g + 8 * (e >> 1), j = cc % 64 + 2 * t + (e & 1);
                if (i < rows && j < cols) c[(size_t)j * ld + i] -= acc[mi][ni][e];
            }
        }
    }
}

// The block row of LU step k: A(k, n) <- W A(k, n), n > k, with W the
// inverse of the unit-lower diagonal tile (64 x 64 FP32 tiles): two tile
// columns per CTA of four warps, the tiles copied into shared memory before
// they are overwritten.
__global__ void __launch_bounds__(128)
k_lu_rowsolve(plasma_desc_t A, int k, const float *W, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) float lg_raw[];
    float *As = lg_raw;                        // [64][LG_LDA]  W
    float *Bs = lg_raw + 64 * LG_LDA;          // [128][LG_LDB] A(k, n..n+1), [j][k]
    if (plasma_failed(st)) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int n0 = k + 1 + 2 * blockIdx.x;
    const int kb = plasma_tile_mview(A, k);
    lg_stage(As, LG_LDA, W + (size_t)k * 64 * 64, 64, kb, kb, tid, 128);
    for (int h = 0; h < 2; h++) {
        const int n = n0 + h;
        const bool nv = n < A.nt;
        lg_stage(Bs + 64 * h * LG_LDB, LG_LDB,
                 nv ? (const float *)plasma_tile_addr(A, k, n) : nullptr,
                 plasma_tile_mmain(A, k), kb, nv ? plasma_tile_nview(A, n) : 0, tid, 128);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    float acc[4][4][4];
    lg_product(As, Bs, 0, warp * 32, g, t, acc);
    const int ld = plasma_tile_mmain(A, k);
#pragma unroll
    for (int ni = 0; ni < 4; ni++) {
        const int cc = warp * 32 + ni * 8;
        const int n = n0 + cc / 64;
        if (n >= A.nt) continue;
        const int cols = plasma_tile_nview(A, n);
        float *c = (float *)plasma_tile_addr(A, k, n);
#pragma unroll
        for (int mi = 0; mi < 4; mi++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = mi * 16 + g + 8 * (e >> 1), j = cc % 64 + 2 * t + (e & 1);
                if (i < kb && j < cols) c[(size_t)j * ld + i] = acc[mi][ni][e];
            }
    }
}

// Partial row sums of a general tile matrix over GV_SPLIT ranges of tile
// columns: part[s][i] = sum over the range s of A(i, c) x[c] (ABS: |A(i, c)|,
// x unused), one CTA per (tile row, range), threads over rows and column
// groups (coalesced along the column-major tiles); k_gemv_finish adds the
// ranges in a fixed order.
constexpr int GV_SPLIT = 16;

template <typename T, bool ABS>
__global__ void __launch_bounds__(256)
k_gemv_part(plasma_desc_t A, const T *x, double *part, const plasma_devstat_t *st)
{
    __shared__ double red[256];
    if (plasma_failed(st)) return;
    const int m = blockIdx.x, sp = blockIdx.y, tid = threadIdx.x;
    const int rows = plasma_tile_mview(A, m), ld = plasma_tile_mmain(A, m);
    const int G = A.mb >= 256 ? 1 : 256 / A.mb;          // column groups
    const int RB = A.mb >= 256 ? 256 : A.mb;             // rows per pass
    const int g = tid / RB, r = tid % RB;
    const int per = (A.nt + GV_SPLIT - 1) / GV_SPLIT;
    const int n0 = sp * per, n1 = min(A.nt, n0 + per);
    for (int rb = 0; rb < rows; rb += RB) {
        double acc = 0.0;
        const int row = rb + r;
        if (g < G && row < rows) {
            for (int n = n0; n < n1; n++) {
                const T *t = (const T *)plasma_tile_addr(A, m, n) + row;
                const int w = plasma_tile_nview(A, n);
                for (int c = g; c < w; c += G) {
                    const double v = (double)t[(size_t)c * ld];
                    acc += ABS ? fabs(v) : v * (double)x[(size_t)n * A.nb + c];
                }
            }
        }
        red[tid] = acc;
        __syncthreads();
        if (tid < RB && rb + tid < rows) {
            double sum = 0.0;
            for (int q = 0; q < G; q++) sum += red[q * RB + tid];
            part[(size_t)sp * A.m + (size_t)m * A.mb + rb + tid] = sum;
        }
        __syncthreads();
    }
}

// ABS: *out = max_i sum_s part[s][i] (atomic max of the bit patterns of
// non-negative doubles; *out zeroed by the caller); else y[i] -= sum_s.
template <typename T, bool ABS>
__global__ void __launch_bounds__(256)
k_gemv_finish(const double *part, int n, T *y, double *out, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sum = 0.0;
    for (int q = 0; q < GV_SPLIT; q++) sum += part[(size_t)q * n + i];
    if (ABS)
        atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(sum));
    else
        y[i] = (T)((double)y[i] - sum);
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

// ---------------------------------------------------------------------------
// The panel of tile column k (kb <= 64 columns) in one launch, resident in
// the shared memory of a cluster of CL_CTAS CTAs: CTA c holds panel rows
// [c R, (c+1) R), column-major.  Per column j: every CTA finds its candidate
// (the first largest magnitude among its rows >= j) and publishes it with a
// copy of that row -- and, if it holds row j, a copy of row j -- in a slot of
// its shared memory (two slots, alternating with j); one cluster barrier;
// every CTA reads the candidates, picks the pivot p (first largest, as
// LAPACK's idamax), takes the pivot row from p's owner, and the owners of
// rows j and p write the swapped rows; then the rows below j are scaled and
// take the rank-1 update inside the sub-block of CL_IB columns.  After a
// sub-block its rows are published (one more cluster barrier), every CTA
// solves them with the unit-lower sub-block diagonal (U12 = L11^-1 A12) and
// updates its rows below (A22 -= L21 U12).  Every CTA runs the same barrier
// sequence; a zero pivot records info (the first one, as k_lu_pivot) and
// the factorization goes on without scaling that column.
// ---------------------------------------------------------------------------
constexpr int CL_CTAS = 8;
constexpr int CL_THREADS = 256;
constexpr int CL_KB = 64;
constexpr int CL_IB = 16;

template <typename T> struct ClLayout {
    // shared memory after the panel (R x CL_KB): two publication slots of a
    // candidate row and a row-j copy, the sub-block rows published and the
    // local copy of them, the pivot row, the row j copy read back
    static constexpr int EXTRA = (2 * 2 * CL_KB + 2 * CL_IB * CL_KB + 2 * CL_KB) * sizeof(T) +
                                 2 * (sizeof(T) + sizeof(int)) + 64 * (sizeof(T) + 4) + 64;
    static constexpr int MAX_SMEM = 227 * 1024 - 256;      // room for the static part
    static constexpr int MAX_R = (MAX_SMEM - EXTRA) / (CL_KB * (int)sizeof(T));
};

__device__ __forceinline__ uint32_t cl_addr(const void *p, uint32_t rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ float cl_ld(uint32_t a, float)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ double cl_ld(uint32_t a, double)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ int cl_ld_int(uint32_t a)
{
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void cl_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <typename T>
__global__ void __cluster_dims__(CL_CTAS, 1, 1) __launch_bounds__(CL_THREADS, 1)
k_lu_panel_cl(plasma_desc_t A, int k, int kb, int R, int *ipiv, plasma_devstat_t *st,
              int call)
{
    extern __shared__ __align__(16) unsigned char cl_raw[];
    T *P = reinterpret_cast<T *>(cl_raw);                  // [CL_KB][R]
    T *pub_row = P + (size_t)CL_KB * R;                    // [2][2][CL_KB]
    T *blk = pub_row + 4 * CL_KB;                          // [CL_IB][CL_KB] published
    T *u12 = blk + CL_IB * CL_KB;                          // [CL_IB][CL_KB] local copy
    T *prow = u12 + CL_IB * CL_KB;                         // [CL_KB]
    T *rowj = prow + CL_KB;                                // [CL_KB]
    T *pub_val = rowj + CL_KB;                             // [2]
    int *pub_idx = reinterpret_cast<int *>(pub_val + 2);   // [2]
    T *red_v = reinterpret_cast<T *>(pub_idx + 2);         // [CL_THREADS / 32]
    int *red_i = reinterpret_cast<int *>(red_v + CL_THREADS / 32);
    __shared__ int flag_s, piv_s, bi_s;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t me;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(me));
    const int mb = A.mb, d0 = k * mb;
    const int M = A.m - d0;
    const int row0 = (int)me * R;                          // first panel row of this CTA
    const int nown = max(0, min(R, M - row0));             // rows held here

    // a uniform start: everyone follows rank 0's reading of the status
    if (tid == 0) flag_s = plasma_failed(st) ? 1 : 0;
    cl_sync();
    const int failed = cl_ld_int(cl_addr(&flag_s, 0));
    cl_sync();                     // rank 0 stays until everyone has read it
    if (failed) return;

    // a thread per row: the row's kb entries are ld apart in its tile, and
    // a warp's rows are adjacent (coalesced); 16 loads in flight
    for (int r = tid; r < R; r += CL_THREADS) {
        if (r >= nown) {
            for (int c = 0; c < kb; c++) P[(size_t)c * R + r] = T(0);
            continue;
        }
        const T *src = panel_at<T>(A, k, row0 + r, 0);
        const int ld = plasma_tile_mmain(A, k + (row0 + r) / mb);
        for (int c0 = 0; c0 < kb; c0 += 16) {
            T v[16];
#pragma unroll
            for (int q = 0; q < 16; q++) v[q] = c0 + q < kb ? src[(size_t)(c0 + q) * ld] : T(0);
#pragma unroll
            for (int q = 0; q < 16; q++)
                if (c0 + q < kb) P[(size_t)(c0 + q) * R + r] = v[q];
        }
    }
    __syncthreads();

    for (int s0 = 0; s0 < kb; s0 += CL_IB) {
        const int ce = min(kb, s0 + CL_IB);
        // this thread's candidate for the next column: found by a scan at the
        // start of a sub-block, then by each column's rank-1 update
        T bv = T(-1);
        int bi = INT_MAX;
        for (int r = tid; r < nown; r += CL_THREADS)
            if (row0 + r >= s0) max_pick(bv, bi, (T)fabs(P[(size_t)s0 * R + r]), row0 + r);
        for (int j = s0; j < ce; j++) {
            const int par = j & 1;
            T *slot = pub_row + par * 2 * CL_KB;
            // 1. this CTA's candidate for column j and its row
            block_best(bv, bi, red_v, red_i);
            if (tid == 0) {
                pub_val[par] = bv;
                pub_idx[par] = bi;
                bi_s = bi;
            }
            __syncthreads();
            const int cb = bi_s;
            const int rj = j - row0;
            for (int c = tid; c < kb; c += CL_THREADS) {
                slot[c] = cb != INT_MAX ? P[(size_t)c * R + (cb - row0)] : T(0);
                if (rj >= 0 && rj < nown) slot[CL_KB + c] = P[(size_t)c * R + rj];
            }
            cl_sync();
            // 2. the pivot (first largest magnitude over the CTAs'
            // candidates, warp 0) and, in the same round of remote reads,
            // every CTA's candidate row and row j (a thread per column)
            const int cj = j / R;
            T cand[CL_CTAS];
            if (tid < kb) {
#pragma unroll
                for (int q = 0; q < CL_CTAS; q++)
                    cand[q] = cl_ld(cl_addr(&slot[tid], (uint32_t)q), T(0));
                rowj[tid] = cl_ld(cl_addr(&slot[CL_KB + tid], (uint32_t)cj), T(0));
            }
            if (warp == 0) {
                T v = T(-1);
                int i = INT_MAX;
                if (lane < CL_CTAS) {
                    v = cl_ld(cl_addr(&pub_val[par], lane), T(0));
                    i = cl_ld_int(cl_addr(&pub_idx[par], lane));
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    max_pick(v, i, __shfl_xor_sync(0xffffffffu, v, o),
                             __shfl_xor_sync(0xffffffffu, i, o));
                if (lane == 0) piv_s = i == INT_MAX ? j : i;   // a column of NaNs
            }
            __syncthreads();
            const int p = piv_s;
            const int cp = p / R;
            // 3. the pivot row is the candidate row of p's owner
            if (tid < kb) {
                T x = cand[0];
#pragma unroll
                for (int q = 1; q < CL_CTAS; q++)
                    if (q == cp) x = cand[q];
                prow[tid] = x;
            }
            __syncthreads();
            const T piv = prow[j];
            if (me == 0 && tid == 0) {
                ipiv[d0 + j] = d0 + p + 1;
                if (piv == T(0)) plasma_fail(st, d0 + j + 1, call);
            }
            // 4. the swap (a thread per column), then the rows below j:
            // scaled, rank-1 update inside the sub-block, and the candidate
            // for column j+1 on the way
            if (p != j) {
                for (int c = tid; c < kb; c += CL_THREADS) {
                    if (cj == (int)me) P[(size_t)c * R + (j - row0)] = prow[c];
                    if (cp == (int)me) P[(size_t)c * R + (p - row0)] = rowj[c];
                }
                __syncthreads();
            }
            const bool rcp = (T)fabs(piv) >= tiny<T>();
            const T rp = piv != T(0) ? T(1) / piv : T(0);
            bv = T(-1);
            bi = INT_MAX;
            for (int r = tid; r < nown; r += CL_THREADS) {
                const int pr = row0 + r;
                if (pr <= j) continue;
                if (piv != T(0)) {
                    // LAPACK's dgetf2: a reciprocal unless the pivot is tiny
                    T *lr = &P[(size_t)j * R + r];
                    const T l = rcp ? *lr * rp : *lr / piv;
                    *lr = l;
                    for (int c = j + 1; c < ce; c++) P[(size_t)c * R + r] -= l * prow[c];
                }
                if (j + 1 < ce)
                    max_pick(bv, bi, (T)fabs(P[(size_t)(j + 1) * R + r]), pr);
            }
        }
        __syncthreads();
        if (ce >= kb) break;
        // 5. the sub-block's rows to every CTA, U12 = L11^-1 A12, A22 -= L21 U12
        const int nsb = ce - s0;
        for (int e = tid; e < nsb * kb; e += CL_THREADS) {
            const int i = e / kb, c = e % kb, r = s0 + i - row0;
            if (r >= 0 && r < nown) blk[i * CL_KB + c] = P[(size_t)c * R + r];
        }
        cl_sync();
        for (int e = tid; e < nsb * kb; e += CL_THREADS) {
            const int i = e / kb, c = e % kb;
            u12[i * CL_KB + c] = cl_ld(cl_addr(&blk[i * CL_KB + c], (uint32_t)((s0 + i) / R)),
                                       T(0));
        }
        __syncthreads();
        for (int c = ce + tid; c < kb; c += CL_THREADS) {
            for (int i = 1; i < nsb; i++) {
                T v = u12[i * CL_KB + c];
                for (int q = 0; q < i; q++) v -= u12[i * CL_KB + s0 + q] * u12[q * CL_KB + c];
                u12[i * CL_KB + c] = v;
            }
        }
        __syncthreads();
        // rows pr >= ce take A22 -= L21 U12 (nsb = CL_IB here), two rows of
        // a thread at a time so each U12 entry read serves both
        for (int r = tid; r < nown; r += 2 * CL_THREADS) {
            const int r2 = r + CL_THREADS;
            T l[2][CL_IB];
            bool on[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int rr = h ? r2 : r, pr = row0 + rr;
                on[h] = rr < nown && pr >= ce;
                if (rr < nown && pr >= s0 && pr < ce)
                    for (int c = ce; c < kb; c++)
                        P[(size_t)c * R + rr] = u12[(pr - s0) * CL_KB + c];
#pragma unroll
                for (int q = 0; q < CL_IB; q++)
                    l[h][q] = on[h] ? P[(size_t)(s0 + q) * R + rr] : T(0);
            }
            if (!on[0] && !on[1]) continue;
            for (int c = ce; c < kb; c++) {
                T v0 = on[0] ? P[(size_t)c * R + r] : T(0);
                T v1 = on[1] ? P[(size_t)c * R + r2] : T(0);
#pragma unroll
                for (int q = 0; q < CL_IB; q++) {
                    const T u = u12[q * CL_KB + c];
                    v0 -= l[0][q] * u;
                    v1 -= l[1][q] * u;
                }
                if (on[0]) P[(size_t)c * R + r] = v0;
                if (on[1]) P[(size_t)c * R + r2] = v1;
            }
        }
        __syncthreads();
    }
    for (int r = tid; r < nown; r += CL_THREADS) {
        T *dst = panel_at<T>(A, k, row0 + r, 0);
        const int ld = plasma_tile_mmain(A, k + (row0 + r) / mb);
        for (int c = 0; c < kb; c++) dst[(size_t)c * ld] = P[(size_t)c * R + r];
    }
    // no CTA leaves while another may still read its shared memory
    cl_sync();
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
namespace {
// The one-launch cluster panel (k_lu_panel_cl) when the panel fits the
// cluster's shared memory.
template <typename T> bool panel_cluster_ok(int kb, int M)
{
    return kb <= CL_KB && (M + CL_CTAS - 1) / CL_CTAS <= ClLayout<T>::MAX_R;
}

template <typename T>
void panel_cluster(cudaStream_t s, plasma_devstat_t *st, int call, plasma_desc_t A, int k,
                   int kb, int M, int *ipiv)
{
    const int R = (M + CL_CTAS - 1) / CL_CTAS;
    const size_t smem = (size_t)CL_KB * R * sizeof(T) + ClLayout<T>::EXTRA;
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr))
        cudaFuncSetAttribute(k_lu_panel_cl<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ClLayout<T>::MAX_SMEM);
    PLASMA_COUNT_LAUNCH();
    k_lu_panel_cl<T><<<CL_CTAS, CL_THREADS, smem, s>>>(A, k, kb, R, ipiv, st, call);
}
}  // namespace

// The panel of tile column k: the cluster kernel when kb <= 64 and the panel
// fits (PLASMA_LU_CLUSTER=0 turns it off), else the per-column kernels.
extern "C" void plasma_cuda_getrf_panel(cudaStream_t s, plasma_devstat_t *st, int call,
                                        plasma_desc_t A, int k, int *ipiv, void *parts)
{
    const int M = A.m - k * A.mb;
    const int kb = min(plasma_tile_nview(A, k), M);
    if (kb <= 0) return;
    static int cl_env = -1;
    if (cl_env < 0) {
        const char *e = getenv("PLASMA_LU_CLUSTER");
        cl_env = e ? atoi(e) != 0 : 1;
    }
    const bool dp = A.precision == PlasmaRealDouble;
    if (cl_env && (dp ? panel_cluster_ok<double>(kb, M) : panel_cluster_ok<float>(kb, M))) {
        int prof = plasma_prof_begin(s);
        if (dp)
            panel_cluster<double>(s, st, call, A, k, kb, M, ipiv);
        else
            panel_cluster<float>(s, st, call, A, k, kb, M, ipiv);
        plasma_prof_end(prof, s, PLASMA_KCLASS_POTRF,
                        (double)M * kb * kb - (double)kb * kb * kb / 3.0,
                        2.0 * (double)M * kb * plasma_element_size(A.precision));
        return;
    }
    const int G = (M + kRows - 1) / kRows;
    const size_t es = plasma_element_size(A.precision);
    int *pidx = (int *)((char *)parts + (((size_t)G * es + 15) & ~(size_t)15));
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

// The trailing update of LU step k on the tensor cores for 64 x 64 FP32
// tiles; returns 0 (nothing launched) for other tilings.
extern "C" int plasma_cuda_lu_update(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                     int k)
{
    if (A.precision != PlasmaRealFloat || A.mb != 64 || A.nb != 64) return 0;
    const int rt = A.mt - k - 1, ct = A.nt - k - 1;
    if (rt <= 0 || ct <= 0) return 1;
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr))
        cudaFuncSetAttribute(k_lu_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, LG_SMEM);
    PLASMA_COUNT_LAUNCH();
    const double M = A.m - (k + 1) * 64.0, N = A.n - (k + 1) * 64.0;
    int prof = plasma_prof_begin(s);
    dim3 grid((unsigned)((ct + 1) / 2), (unsigned)((rt + 1) / 2));
    k_lu_gemm<<<grid, LG_THREADS, LG_SMEM, s>>>(A, k, st);
    plasma_prof_end(prof, s, PLASMA_KCLASS_UPDATE, 2.0 * M * N * 64.0, 4.0 * (2.0 * M * N));
    return 1;
}

// The block row of LU step k, A(k, n) <- WL_k A(k, n) for n > k (WL: the
// inverses of the unit-lower diagonal tiles, 64 x 64 each); 0 (nothing
// launched) for other tilings.
extern "C" int plasma_cuda_lu_rowsolve(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                       int k, const void *WL)
{
    if (A.precision != PlasmaRealFloat || A.mb != 64 || A.nb != 64) return 0;
    const int ct = A.nt - k - 1;
    if (ct <= 0) return 1;
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr))
        cudaFuncSetAttribute(k_lu_rowsolve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             LG_SMEM);
    PLASMA_COUNT_LAUNCH();
    k_lu_rowsolve<<<(unsigned)((ct + 1) / 2), 128, LG_SMEM, s>>>(A, k, (const float *)WL, st);
    return 1;
}

// perm (device, n ints) <- the composition of the interchanges ipiv[0 .. n);
// 0 (nothing launched) when n is too large for one CTA's shared memory.
extern "C" int plasma_cuda_lu_perm(cudaStream_t s, plasma_devstat_t *st, const int *ipiv,
                                   int n, int *perm)
{
    const size_t bytes = 2 * sizeof(int) * (size_t)n;
    if (n <= 0 || bytes > 200 * 1024) return 0;
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr))
        cudaFuncSetAttribute(k_ipiv_perm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    PLASMA_COUNT_LAUNCH();
    k_ipiv_perm<<<1, 256, bytes, s>>>(ipiv, n, perm, st);
    return 1;
}

// The rows of column col of D reordered by perm (plasma_cuda_lu_perm): the
// interchanges applied to a right-hand side.  0 when n is too large.
extern "C" int plasma_cuda_permute_vec(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                                       int col, const int *perm, int n)
{
    const size_t bytes = plasma_element_size(D.precision) * (size_t)n;
    if (n <= 0 || bytes > 200 * 1024) return 0;
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_permute_vec<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_permute_vec<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    }
    PLASMA_COUNT_LAUNCH();
    if (D.precision == PlasmaRealDouble)
        k_permute_vec<double><<<1, 1024, bytes, s>>>(D, col, perm, n, st);
    else
        k_permute_vec<float><<<1, 1024, bytes, s>>>(D, col, perm, n, st);
    return 1;
}

// Largest panel height of the cluster panel kernel for 64-wide tiles.
extern "C" int plasma_cuda_getrf_cluster_rows(int precision)
{
    return CL_CTAS * (precision == PlasmaRealDouble ? ClLayout<double>::MAX_R
                                                    : ClLayout<float>::MAX_R);
}

extern "C" size_t plasma_cuda_getrf_parts_bytes(plasma_desc_t A)
{
    const size_t G = (size_t)(A.m + kRows - 1) / kRows;
    return ((G * 8 + 15) & ~(size_t)15) + G * sizeof(int) + 64;
}

extern "C" void plasma_cuda_laswp(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                                  const int *ipiv, int j0, int j1, int c0, int c1)
{
    if (j1 <= j0 || c1 <= c0) return;
    const bool dp = D.precision == PlasmaRealDouble;
    const size_t es = plasma_element_size(D.precision);
    // one column, every interchange: in shared memory
    const size_t vbytes = (size_t)(j1) * (es + sizeof(int));
    if (j0 == 0 && c1 - c0 == 1 && vbytes <= 200 * 1024) {
        static unsigned long long attr = 0;
        if (plasma_first_on_device(&attr)) {
            cudaFuncSetAttribute(k_laswp_vec<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(k_laswp_vec<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        PLASMA_COUNT_LAUNCH();
        if (dp)
            k_laswp_vec<double><<<1, 256, vbytes, s>>>(D, c0, ipiv, j1, st);
        else
            k_laswp_vec<float><<<1, 256, vbytes, s>>>(D, c0, ipiv, j1, st);
        return;
    }
    // up to 64 rows at a time: the block kernel
    plasma_cuda_laswp_skip(s, st, D, ipiv, j0, j1, c0, c1, c1, c1);
}

// As plasma_cuda_laswp on the columns [c0, c1) except [skip0, skip1), in
// one launch per 64 rows.
extern "C" void plasma_cuda_laswp_skip(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                                       const int *ipiv, int j0, int j1, int c0, int c1,
                                       int skip0, int skip1)
{
    skip0 = max(skip0, c0);
    skip1 = max(skip0, min(skip1, c1));
    const int ncols = c1 - c0 - (skip1 - skip0);
    if (j1 <= j0 || ncols <= 0) return;
    const bool dp = D.precision == PlasmaRealDouble;
    const unsigned grid = (unsigned)((ncols + LW_COLS - 1) / LW_COLS);
    for (int b = j0; b < j1; b += 64) {
        const int nj = min(64, j1 - b);
        PLASMA_COUNT_LAUNCH();
        if (dp)
            k_laswp_rows<double><<<grid, 32 * LW_WARPS, 0, s>>>(D, ipiv, b, nj, c0, c1, skip0,
                                                               skip1, st);
        else
            k_laswp_rows<float><<<grid, 32 * LW_WARPS, 0, s>>>(D, ipiv, b, nj, c0, c1, skip0,
                                                              skip1, st);
    }
}

extern "C" void plasma_cuda_trtri_lu(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                     int k0, int k1, void *WL, void *WU)
{
    if (k1 <= k0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.mb == 64 && A.nb == 64) {
        static unsigned long long attr = 0;
        if (plasma_first_on_device(&attr)) {
            cudaFuncSetAttribute(k_trtri_lu64<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, LU_INV_SMEM);
            cudaFuncSetAttribute(k_trtri_lu64<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, LU_INV_SMEM);
        }
        if (A.precision == PlasmaRealDouble)
            k_trtri_lu64<double><<<2 * (k1 - k0), 256, LU_INV_SMEM, s>>>(
                A, k0, (double *)WL, (double *)WU, st);
        else
            k_trtri_lu64<float><<<2 * (k1 - k0), 256, LU_INV_SMEM, s>>>(
                A, k0, (float *)WL, (float *)WU, st);
        return;
    }
    if (A.precision == PlasmaRealDouble)
        k_trtri_lu<double><<<k1 - k0, 512, 0, s>>>(A, k0, (double *)WL, (double *)WU, st);
    else
        k_trtri_lu<float><<<k1 - k0, 512, 0, s>>>(A, k0, (float *)WL, (float *)WU, st);
}

extern "C" size_t plasma_cuda_gemv_part_bytes(plasma_desc_t A)
{
    return (size_t)GV_SPLIT * A.m * sizeof(double);
}

// ||A||_inf of a general tile matrix into *dnorm; `part`: device scratch
// of plasma_cuda_gemv_part_bytes(A) bytes.
extern "C" void plasma_cuda_lange_inf(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                      double *dnorm, double *part)
{
    cudaMemsetAsync(dnorm, 0, sizeof(double), s);
    if (A.m == 0 || A.n == 0) return;
    PLASMA_COUNT_LAUNCH();
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)A.mt, GV_SPLIT);
    const unsigned g2 = (unsigned)((A.m + 255) / 256);
    if (A.precision == PlasmaRealDouble) {
        k_gemv_part<double, true><<<grid, 256, 0, s>>>(A, nullptr, part, st);
        k_gemv_finish<double, true><<<g2, 256, 0, s>>>(part, A.m, nullptr, dnorm, st);
    } else {
        k_gemv_part<float, true><<<grid, 256, 0, s>>>(A, nullptr, part, st);
        k_gemv_finish<float, true><<<g2, 256, 0, s>>>(part, A.m, nullptr, dnorm, st);
    }
}

// y -= A x for one right-hand side: x and y contiguous vectors of the
// precision of A (the single columns of n x 1 tile matrices); `part` as for
// plasma_cuda_lange_inf.  Sums in FP64.
extern "C" void plasma_cuda_gemv_sub(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                     const void *x, void *y, double *part)
{
    if (A.m == 0 || A.n == 0) return;
    PLASMA_COUNT_LAUNCH();
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)A.mt, GV_SPLIT);
    const unsigned g2 = (unsigned)((A.m + 255) / 256);
    if (A.precision == PlasmaRealDouble) {
        k_gemv_part<double, false><<<grid, 256, 0, s>>>(A, (const double *)x, part, st);
        k_gemv_finish<double, false><<<g2, 256, 0, s>>>(part, A.m, (double *)y, nullptr, st);
    } else {
        k_gemv_part<float, false><<<grid, 256, 0, s>>>(A, (const float *)x, part, st);
        k_gemv_finish<float, false><<<g2, 256, 0, s>>>(part, A.m, (float *)y, nullptr, st);
    }
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
