// potrf_tile.cu -- the serial part of every Cholesky step.
//
//  * k_potrf_tile: Cholesky of the diagonal tile (k,k), one CTA, the tile
//    streamed through shared memory in 32-column panels (right-looking inside
//    the tile).  Replaces plasma_core_dpotrf -> LAPACKE_dpotrf_work
//    (core_blas/core_zpotrf.c:54-82): same info rule -- the first column j
//    whose pivot is not > 0 (or NaN) gives info = iinfo + j (1-based), which
//    the reference forms as A.nb*k + info (compute/pzpotrf.c:44).
//  * k_trsm_panel: A(m,k) <- A(m,k) L_kk^{-T} for all m > k in one launch
//    (the nt-k-1 plasma_core_dtrsm tasks of compute/pzpotrf.c:50-56).  Each
//    CTA keeps 32 rows of one tile in shared memory and eliminates column by
//    column; L_kk is read from L2.
//  * k_trtri_tiles: inverses of all diagonal tiles of a factor, one CTA per
//    tile, used by the blocked triangular solves of potrs.
#include "common.cuh"

namespace {

constexpr int kIB = 32;          // panel width inside the diagonal tile
constexpr int kPotrfThreads = 512;

template <typename T>
__device__ __forceinline__ T ld_view(const TileView<T> &v, int i, int j)
{
    return v.at(i, j);
}

template <typename T>
__global__ void __launch_bounds__(kPotrfThreads)
k_potrf_tile(plasma_desc_t A, int uplo, int k, int iinfo,
             plasma_devstat_t *st, int call)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *P = reinterpret_cast<T *>(smem_raw);   // [n][kIB+1] row-major panel
    __shared__ int failed;

    if (plasma_failed(st)) return;
    TileView<T> L = tile_view<T>(A, uplo, k, k);
    const int n = L.rows;
    const int ldp = kIB + 1;
    const int tid = threadIdx.x;
    if (tid == 0) failed = 0;

    for (int j0 = 0; j0 < n; j0 += kIB) {
        const int jb = min(kIB, n - j0);
        const int rows = n - j0;
        __syncthreads();
        // load panel P[r][c] = L(j0+r, j0+c), lower part only
        for (int e = tid; e < rows * jb; e += kPotrfThreads) {
            int r = e % rows, c = e / rows;
            P[r * ldp + c] = r >= c ? L.at(j0 + r, j0 + c) : T(0);
        }
        __syncthreads();
        // unblocked right-looking factorisation of the tall panel
        for (int c = 0; c < jb; c++) {
            T d = P[c * ldp + c];
            if (!(d > T(0))) {
                if (tid == 0) {
                    failed = 1;
                    plasma_fail(st, iinfo + j0 + c + 1, call);
                }
                __syncthreads();
                return;
            }
            d = sqrt(d);
            T rd = T(1) / d;
            __syncthreads();
            for (int r = c + tid; r < rows; r += kPotrfThreads)
                P[r * ldp + c] = (r == c) ? d : P[r * ldp + c] * rd;
            __syncthreads();
            for (int r = c + 1 + tid; r < rows; r += kPotrfThreads) {
                T lrc = P[r * ldp + c];
                int cmax = min(jb - 1, r);
                for (int c2 = c + 1; c2 <= cmax; c2++)
                    P[r * ldp + c2] -= lrc * P[c2 * ldp + c];
            }
            __syncthreads();
        }
        // store the panel (lower part; the strict upper part of the
        // diagonal tile is never written, as LAPACK leaves it untouched)
        for (int e = tid; e < rows * jb; e += kPotrfThreads) {
            int r = e % rows, c = e / rows;
            if (r >= c) L.at(j0 + r, j0 + c) = P[r * ldp + c];
        }
        // trailing update of the rest of the tile:
        //   L(i,j) -= sum_c P[i-j0][c] * P[j-j0][c], j0+jb <= j <= i < n
        const int t0 = j0 + jb;
        const int tr = n - t0;
        if (tr > 0) {
            __syncthreads();
            const int nbk = (tr + 3) / 4;
            const int npairs = nbk * (nbk + 1) / 2;
            // pair index -> (bi, bj), column-major over the lower triangle
            int p = tid, bj = 0, base = 0;
            while (p < npairs) {
                while (p - base >= nbk - bj) { base += nbk - bj; bj++; }
                int bi = bj + (p - base);
                int i0 = bi * 4, jj0 = bj * 4;
                T acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 4; b++) acc[a][b] = T(0);
                for (int c = 0; c < jb; c++) {
                    T x[4], y[4];
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        int ri = jb + i0 + a, rj = jb + jj0 + a;
                        x[a] = ri < rows ? P[ri * ldp + c] : T(0);
                        y[a] = rj < rows ? P[rj * ldp + c] : T(0);
                    }
#pragma unroll
                    for (int a = 0; a < 4; a++)
#pragma unroll
                        for (int b = 0; b < 4; b++) acc[a][b] += x[a] * y[b];
                }
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    int j = t0 + jj0 + b;
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        int i = t0 + i0 + a;
                        if (i < n && j < n && i >= j)
                            L.at(i, j) -= acc[a][b];
                    }
                }
                p += kPotrfThreads;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Panel solve: X L^T = A(m,k) for the rows of every tile m in [mlo, mhi).
// grid.x = tile index, grid.y = 32-row block of that tile.
// ---------------------------------------------------------------------------
constexpr int kTrsmRows = 32;
constexpr int kTrsmThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kTrsmThreads)
k_trsm_panel(plasma_desc_t A, int uplo, int k, int mlo, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (plasma_failed(st)) return;
    const int m = mlo + blockIdx.x;
    TileView<T> L = tile_view<T>(A, uplo, k, k);
    TileView<T> B = tile_view<T>(A, uplo, m, k);
    const int n = L.rows;
    const int r0 = blockIdx.y * kTrsmRows;
    const int nr = min(kTrsmRows, B.rows - r0);
    if (nr <= 0) return;
    const int ldx = n + 1;
    T *X = reinterpret_cast<T *>(smem_raw);    // [kTrsmRows][n+1]
    const int tid = threadIdx.x;
    const int r = tid % kTrsmRows;             // row owned
    const int g = tid / kTrsmRows;             // column group (8 groups)
    constexpr int kGroups = kTrsmThreads / kTrsmRows;

    for (int e = tid; e < nr * n; e += kTrsmThreads) {
        int rr = e % nr, c = e / nr;
        X[rr * ldx + c] = B.at(r0 + rr, c);
    }
    __syncthreads();
    for (int c = 0; c < n; c++) {
        // x_c = x_c / L(c,c), then x_c2 -= x_c L(c2,c) for c2 > c
        T lcc = L.at(c, c);
        T xc = X[r * ldx + c] / lcc;
        __syncthreads();
        if (g == 0) X[r * ldx + c] = xc;
        for (int c2 = c + 1 + g; c2 < n; c2 += kGroups)
            X[r * ldx + c2] -= xc * L.at(c2, c);
        __syncthreads();
    }
    for (int e = tid; e < nr * n; e += kTrsmThreads) {
        int rr = e % nr, c = e / nr;
        B.at(r0 + rr, c) = X[rr * ldx + c];
    }
}

// ---------------------------------------------------------------------------
// W_k = inv(L_kk) for every diagonal tile k (lower logical view), written to
// a dense workspace of nt tiles of nb x nb, column-major, ld = nb.
// Solves L W = I a block of 32 columns at a time, right-looking.
// ---------------------------------------------------------------------------
constexpr int kInvCols = 32;
constexpr int kInvThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kInvThreads)
k_trtri_tiles(plasma_desc_t A, int uplo, T *W, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (plasma_failed(st)) return;
    const int k = blockIdx.x;
    TileView<T> L = tile_view<T>(A, uplo, k, k);
    const int n = L.rows;
    const int nb = A.mb;
    T *Wk = W + (size_t)k * nb * nb;
    T *S = reinterpret_cast<T *>(smem_raw);    // [n][kInvCols+1]
    const int lds = kInvCols + 1;
    const int tid = threadIdx.x;
    for (int c0 = 0; c0 < n; c0 += kInvCols) {
        const int cb = min(kInvCols, n - c0);
        __syncthreads();
        for (int e = tid; e < n * kInvCols; e += kInvThreads) {
            int rr = e % n, c = e / n;
            S[rr * lds + c] = (rr == c0 + c) ? T(1) : T(0);
        }
        __syncthreads();
        for (int j = c0; j < n; j++) {
            T rjj = T(1) / L.at(j, j);
            // scale row j
            if (tid < cb) S[j * lds + tid] *= rjj;
            __syncthreads();
            // rows below j
            for (int e = tid; e < (n - j - 1) * cb; e += kInvThreads) {
                int rr = j + 1 + e / cb, c = e % cb;
                S[rr * lds + c] -= L.at(rr, j) * S[j * lds + c];
            }
            __syncthreads();
        }
        for (int e = tid; e < n * cb; e += kInvThreads) {
            int rr = e % n, c = e / n;
            Wk[(size_t)(c0 + c) * nb + rr] = S[rr * lds + c];
        }
    }
}

template <typename T>
void launch_potrf_tile(cudaStream_t s, plasma_devstat_t *st, int call,
                       int uplo, const plasma_desc_t &A, int k, int iinfo)
{
    int n = plasma_tile_mview(A, k);
    size_t smem = (size_t)n * (kIB + 1) * sizeof(T);
    static unsigned long long attr_set = 0;
    if (plasma_first_on_device(&attr_set)) {
        cudaFuncSetAttribute(k_potrf_tile<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    }
    k_potrf_tile<T><<<1, kPotrfThreads, smem, s>>>(A, uplo, k, iinfo, st, call);
}

template <typename T>
void launch_trsm_panel(cudaStream_t s, plasma_devstat_t *st, int uplo,
                       const plasma_desc_t &A, int k, int mlo, int mhi)
{
    int n = plasma_tile_mview(A, k);
    size_t smem = (size_t)kTrsmRows * (n + 1) * sizeof(T);
    static unsigned long long attr_set = 0;
    if (plasma_first_on_device(&attr_set)) {
        cudaFuncSetAttribute(k_trsm_panel<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    }
    dim3 grid((unsigned)(mhi - mlo), (unsigned)ceil_div(A.mb, kTrsmRows));
    k_trsm_panel<T><<<grid, kTrsmThreads, smem, s>>>(A, uplo, k, mlo, st);
}

template <typename T>
void launch_trtri(cudaStream_t s, plasma_devstat_t *st, int uplo,
                  const plasma_desc_t &A, T *W)
{
    size_t smem = (size_t)A.mb * (kInvCols + 1) * sizeof(T);
    static unsigned long long attr_set = 0;
    if (plasma_first_on_device(&attr_set)) {
        cudaFuncSetAttribute(k_trtri_tiles<T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    }
    k_trtri_tiles<T><<<A.mt, kInvThreads, smem, s>>>(A, uplo, W, st);
}

}  // namespace

extern "C" int plasma_cuda_potrf_diag_fast(cudaStream_t s, plasma_devstat_t *st,
                                          int call, plasma_enum_t uplo,
                                          plasma_desc_t A, int k, int iinfo);
extern "C" int plasma_cuda_trsm_panel_fast(cudaStream_t s, plasma_devstat_t *st,
                                          plasma_enum_t uplo, plasma_desc_t A,
                                          int k, int mlo, int mhi);

extern "C" void plasma_cuda_potrf_tile(cudaStream_t s, plasma_devstat_t *st,
                                       int call, plasma_enum_t uplo,
                                       plasma_desc_t A, int k, int iinfo,
                                       void *winv)
{
    (void)winv;
    if (plasma_cuda_potrf_diag_fast(s, st, call, uplo, A, k, iinfo))
        return;
    PLASMA_COUNT_LAUNCH();
    double nk = plasma_tile_mview(A, k);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        launch_potrf_tile<double>(s, st, call, uplo, A, k, iinfo);
    else
        launch_potrf_tile<float>(s, st, call, uplo, A, k, iinfo);
    plasma_prof_end(prof, s, PLASMA_KCLASS_POTRF, nk * nk * nk / 3.0,
                    nk * nk * plasma_element_size(A.precision));
}

extern "C" void plasma_cuda_trsm_panel(cudaStream_t s, plasma_devstat_t *st,
                                       plasma_enum_t uplo, plasma_desc_t A,
                                       int k, int mlo, int mhi,
                                       const void *winv)
{
    (void)winv;
    if (mhi <= mlo) return;
    if (plasma_cuda_trsm_panel_fast(s, st, uplo, A, k, mlo, mhi))
        return;
    PLASMA_COUNT_LAUNCH();
    double nk = plasma_tile_mview(A, k), rows = 0;
    for (int m = mlo; m < mhi; m++) rows += plasma_tile_mview(A, m);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        launch_trsm_panel<double>(s, st, uplo, A, k, mlo, mhi);
    else
        launch_trsm_panel<float>(s, st, uplo, A, k, mlo, mhi);
    plasma_prof_end(prof, s, PLASMA_KCLASS_TRSM, rows * nk * nk,
                    2.0 * rows * nk * plasma_element_size(A.precision));
}

extern "C" void plasma_cuda_trtri_tiles(cudaStream_t s, plasma_devstat_t *st,
                                        plasma_enum_t uplo, plasma_desc_t A,
                                        void *W)
{
    if (A.mt == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        launch_trtri<double>(s, st, uplo, A, (double *)W);
    else
        launch_trtri<float>(s, st, uplo, A, (float *)W);
}
