// solve.cu -- blocked triangular solves with a tile Cholesky factor.
//
// potrs = two sweeps of plasma_pdtrsm (compute/zpotrs.c:270-282), Left/Lower
// NoTrans then Trans (compute/pztrsm.c:113-177); upper storage solves with
// U^T then U, which on the logical lower view (L = U^T) is the same pair.
// Each tile step of a sweep is two launches:
//   diag  : B(k,:) <- W_k B(k,:)      (W_k = inv(L_kk), precomputed for all
//                                      k by k_trtri_tiles; replaces the
//                                      per-tile trsm task)
//   update: B(m,:) -= L(m,k) B(k,:)   for every m below k (forward) or
//           B(m,:) -= L(k,m)^T B(k,:) for every m above k (backward)
//                                     (the gemm tasks of pztrsm.c:131-141).
// The sweeps are HBM bound: each reads the triangle of the factor once.
#include "common.cuh"

#include <string.h>

namespace {

constexpr int kCols = 16;        // right-hand sides per CTA
constexpr int kThreads = 256;

// out(i, 0:kCols) = sum over c in [cb, ce) of row[c] * Ys[c][0:kCols] for a
// row of the operator that is contiguous in memory, one warp per row: the
// lanes stride along the row (coalesced) and the partial sums are reduced
// across the warp; lane 0 ends with the sums.
template <typename T>
__device__ __forceinline__ void warp_row(const T *row, int cb, int ce,
                                         const T (*Ys)[kCols + 1], T (&acc)[kCols])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < kCols; j++) acc[j] = T(0);
    for (int c = cb + lane; c < ce; c += 32) {
        const T v = row[c];
#pragma unroll
        for (int j = 0; j < kCols; j++) acc[j] += v * Ys[c][j];
    }
#pragma unroll
    for (int j = 0; j < kCols; j++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
}

// out(k) = op(W_k) * B(k, chunk), op = identity (forward) or transpose.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_diag_apply(plasma_desc_t B, int k, const T *W, int nbw, int trans,
             const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T (*Bs)[kCols + 1] = reinterpret_cast<T (*)[kCols + 1]>(smem_raw);
    if (plasma_failed(st)) return;
    const int n = blockIdx.x;
    const int c0 = blockIdx.y * kCols;
    const int rows = plasma_tile_mview(B, k);
    const int cols = min(kCols, plasma_tile_nview(B, n) - c0);
    if (cols <= 0) return;
    T *b = (T *)plasma_tile_addr(B, k, n);
    const int ldb = plasma_tile_mmain(B, k);
    const T *w = W + (size_t)k * nbw * nbw;
    for (int e = threadIdx.x; e < rows * cols; e += kThreads) {
        int r = e % rows, c = e / rows;
        Bs[r][c] = b[(size_t)(c0 + c) * ldb + r];
    }
    __syncthreads();
    if (trans) {
        // backward: out_i = sum_{c >= i} W(c,i) B(c,:); column i of W_k is
        // contiguous, so a warp per row
        for (int i = threadIdx.x >> 5; i < rows; i += kThreads / 32) {
            T acc[kCols];
            warp_row(w + (size_t)i * nbw, i, rows, Bs, acc);
            if ((threadIdx.x & 31) == 0) {
#pragma unroll
                for (int j = 0; j < kCols; j++)
                    if (j < cols) b[(size_t)(c0 + j) * ldb + i] = acc[j];
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < rows; i += kThreads) {
        T acc[kCols];
#pragma unroll
        for (int j = 0; j < kCols; j++) acc[j] = T(0);
        // forward: out_i = sum_{c <= i} W(i,c) B(c,:), W_k lower, coalesced
        // across the threads' rows
        for (int c = 0; c <= i; c++) {
            T wv = w[(size_t)c * nbw + i];
#pragma unroll
            for (int j = 0; j < kCols; j++) acc[j] += wv * Bs[c][j];
        }
#pragma unroll
        for (int j = 0; j < kCols; j++)
            if (j < cols) b[(size_t)(c0 + j) * ldb + i] = acc[j];
    }
}

// B(m, chunk) -= op(L) * B(k, chunk) for the tiles m in [mlo, mhi)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_solve_update(plasma_desc_t A, int uplo, plasma_desc_t B, int k, int mlo,
               int trans, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T (*Ys)[kCols + 1] = reinterpret_cast<T (*)[kCols + 1]>(smem_raw);
    if (plasma_failed(st)) return;
    const int m = mlo + blockIdx.x;
    const int n = blockIdx.y;
    const int c0 = blockIdx.z * kCols;
    const int cols = min(kCols, plasma_tile_nview(B, n) - c0);
    if (cols <= 0) return;
    const int kr = plasma_tile_mview(B, k);
    const int mr = plasma_tile_mview(B, m);
    const T *y = (const T *)plasma_tile_addr(B, k, n);
    const int ldy = plasma_tile_mmain(B, k);
    T *b = (T *)plasma_tile_addr(B, m, n);
    const int ldb = plasma_tile_mmain(B, m);
    for (int e = threadIdx.x; e < kr * cols; e += kThreads) {
        int r = e % kr, c = e / kr;
        Ys[r][c] = y[(size_t)(c0 + c) * ldy + r];
    }
    __syncthreads();
    // forward: L(m,k) (logical lower tile); backward: L(k,m)^T
    TileView<T> L = trans ? tile_view<T>(A, uplo, k, m) : tile_view<T>(A, uplo, m, k);
    if (trans != L.trans) {
        // element (i,c) of the operator is L.p[i*ld + c]: rows contiguous,
        // a warp per row (backward on lower storage, forward on upper)
        for (int i = threadIdx.x >> 5; i < mr; i += kThreads / 32) {
            T acc[kCols];
            warp_row(L.p + (size_t)i * L.ld, 0, kr, Ys, acc);
            if ((threadIdx.x & 31) == 0) {
#pragma unroll
                for (int j = 0; j < kCols; j++)
                    if (j < cols) b[(size_t)(c0 + j) * ldb + i] -= acc[j];
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < mr; i += kThreads) {
        T acc[kCols];
#pragma unroll
        for (int j = 0; j < kCols; j++) acc[j] = T(0);
        for (int c = 0; c < kr; c++) {
            T lv = trans ? L.at(c, i) : L.at(i, c);
#pragma unroll
            for (int j = 0; j < kCols; j++) acc[j] += lv * Ys[c][j];
        }
#pragma unroll
        for (int j = 0; j < kCols; j++)
            if (j < cols) b[(size_t)(c0 + j) * ldb + i] -= acc[j];
    }
}

// kt > 0: A is a band factor whose tile columns hold kt tiles from the
// diagonal down (logical lower view), so step k only reaches tile rows
// [k+1, k+kt) forward and [k-kt+1, k) backward (the reference's band solve,
// compute/pztbsm.c, visits the same tiles).
template <typename T>
void sweep(cudaStream_t s, plasma_devstat_t *st, int uplo, int trans,
           const plasma_desc_t &A, const plasma_desc_t &B, const T *W, int kt)
{
    const int mt = B.mt;
    const int nbw = A.mb;
    const int chunks = ceil_div(B.nb, kCols);
    const size_t smem = (size_t)B.mb * (kCols + 1) * sizeof(T);
    static unsigned long long attr_set = 0;
    if (plasma_first_on_device(&attr_set)) {
        cudaFuncSetAttribute(k_diag_apply<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
        cudaFuncSetAttribute(k_solve_update<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    }
    // many right-hand sides: the update of a step is one tensor-core GEMM on
    // views of the factor and of B (cuda/adjoint.cu, k_gemm_view)
    const bool gemm = B.n >= 64 && A.mb == B.mb;
    for (int step = 0; step < mt; step++) {
        int k = trans ? mt - 1 - step : step;
        PLASMA_COUNT_LAUNCH();
        k_diag_apply<T><<<dim3(B.nt, chunks), kThreads, smem, s>>>(
            B, k, W, nbw, trans, st);
        int mlo = trans ? 0 : k + 1;
        int mhi = trans ? k : mt;
        if (kt > 0) {
            if (trans) mlo = max(0, k - kt + 1);
            else mhi = min(mt, k + kt);
        }
        if (gemm && mhi > mlo &&
            plasma_cuda_sweep_update_mma(s, st, uplo, trans, A, B, k, mlo, mhi)) {
            // square tiles, a multiple of 128: the tensor-core sweep update
            // (cuda/update.cu)
        } else if (gemm && mhi > mlo && kt == 0) {
            const int mb = B.mb, kr = plasma_tile_mview(B, k);
            plasma_view_t lv, bv, cv;
            memset(&lv, 0, sizeof(lv));
            memset(&bv, 0, sizeof(bv));
            memset(&cv, 0, sizeof(cv));
            lv.D = A;
            bv.D = B;
            bv.r0 = k * mb;
            cv.D = B;
            int M;
            if (!trans) {
                // B(k+1.., :) -= L(k+1.., k) B(k, :)
                M = B.m - (k + 1) * mb;
                cv.r0 = (k + 1) * mb;
                if (uplo == PlasmaLower) { lv.r0 = (k + 1) * mb; lv.c0 = k * mb; lv.trans = 0; }
                else { lv.r0 = k * mb; lv.c0 = (k + 1) * mb; lv.trans = 1; }
            } else {
                // B(0..k, :) -= L(k, 0..k)^T B(k, :)
                M = k * mb;
                cv.r0 = 0;
                if (uplo == PlasmaLower) { lv.r0 = k * mb; lv.c0 = 0; lv.trans = 1; }
                else { lv.r0 = 0; lv.c0 = k * mb; lv.trans = 0; }
            }
            plasma_cuda_gemm_view(s, st, M, B.n, kr, -1.0, lv, bv, 1.0, cv, 0, 0);
        } else if (mhi > mlo) {
            PLASMA_COUNT_LAUNCH();
            k_solve_update<T><<<dim3(mhi - mlo, B.nt, chunks), kThreads, smem, s>>>(
                A, uplo, B, k, mlo, trans, st);
        }
    }
}

}  // namespace

extern "C" void plasma_cuda_trtri_tiles(cudaStream_t s, plasma_devstat_t *st,
                                        plasma_enum_t uplo, plasma_desc_t A,
                                        void *W);

// Solves op(L) X = B in place; W holds inv(L_kk) for every k (computed here
// when `have_w` is 0).
extern "C" void plasma_cuda_trsm_sweep(cudaStream_t s, plasma_devstat_t *st,
                                       plasma_enum_t uplo, plasma_enum_t trans,
                                       plasma_desc_t A, plasma_desc_t B,
                                       void *W, int have_w)
{
    if (B.mt == 0 || B.nt == 0) return;
    if (!have_w)
        plasma_cuda_trtri_tiles(s, st, uplo, A, W);
    int t = trans != PlasmaNoTrans;
    const int kt = A.type == PlasmaGeneralBand
                 ? (uplo == PlasmaLower ? A.klt : A.kut) : 0;
    double n = B.m, nrhs = B.n, es = plasma_element_size(A.precision);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        sweep<double>(s, st, uplo, t, A, B, (const double *)W, kt);
    else
        sweep<float>(s, st, uplo, t, A, B, (const float *)W, kt);
    // one triangle of the factor (or its band) read once, B read and
    // written once
    double w = kt > 0 ? fmin(n, (double)kt * A.mb) : n;
    plasma_prof_end(prof, s, PLASMA_KCLASS_SOLVE, n * w * nrhs,
                    es * (n * w / 2.0 + 2.0 * n * nrhs));
}
