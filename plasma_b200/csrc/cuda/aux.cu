// aux.cu -- FP64 kernels of the refinement loop of dsposv.
//
//  * k_lansy_inf: ||A||_inf of the symmetric matrix stored in one triangle
//    (reference compute/pzlansy.c:83-131, Inf-norm = One-norm for symmetric
//    A).  One CTA per tile row; every thread owns one matrix row and sums
//    |a_ij| across the row of stored tiles and the column of mirrored tiles.
//  * k_residual: R = B - A X with A symmetric in one triangle
//    (pzlacpy B->R then pzsymm, compute/zcposv.c:466-467 and
//    compute/pzsymm.c:29-211), fused with the columnwise max-norms of X and
//    R (plasma_pdamax, compute/pdzamax.c:24-79, zcposv.c:471-472).
// Max reductions use atomicMax on the IEEE bit pattern of non-negative
// doubles, which orders like the values; they are order independent, so the
// results are deterministic.
#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kResThreads = 512;   // one matrix row per thread (mb <= 512)
constexpr int kCols = 16;

// Element (i,c) of the logical block (m,k) of the full symmetric matrix.
__device__ __forceinline__ double sym_at(const plasma_desc_t &A, int uplo,
                                         int m, int k, int i, int c)
{
    bool lower = uplo == PlasmaLower;
    if (m == k) {
        const double *p = (const double *)plasma_tile_addr(A, m, m);
        int ld = plasma_tile_mmain(A, m);
        bool stored = lower ? i >= c : i <= c;
        return stored ? p[(size_t)c * ld + i] : p[(size_t)i * ld + c];
    }
    bool direct = lower ? m > k : m < k;
    if (direct) {
        const double *p = (const double *)plasma_tile_addr(A, m, k);
        return p[(size_t)c * plasma_tile_mmain(A, m) + i];
    }
    const double *p = (const double *)plasma_tile_addr(A, k, m);
    return p[(size_t)i * plasma_tile_mmain(A, k) + c];
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
    atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(kThreads)
k_lansy_inf(plasma_desc_t A, int uplo, double *norm, const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int m = blockIdx.x;
    const int rows = plasma_tile_mview(A, m);
    double best = 0.0;
    for (int i = threadIdx.x; i < rows; i += kThreads) {
        double s = 0.0;
        for (int k = 0; k < A.nt; k++) {
            int kc = plasma_tile_nview(A, k);
            for (int c = 0; c < kc; c++)
                s += fabs(sym_at(A, uplo, m, k, i, c));
        }
        best = fmax(best, s);
    }
    // NaN-free reduction of non-negative values
    for (int off = 16; off > 0; off >>= 1)
        best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
    if ((threadIdx.x & 31) == 0)
        atomic_max_nonneg(norm, best);
}

// grid (mt, B.nt, chunks of kCols columns)
__global__ void __launch_bounds__(kResThreads)
k_residual(plasma_desc_t A, int uplo, plasma_desc_t B, plasma_desc_t X,
           plasma_desc_t R, double *xnorm, double *rnorm,
           const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double (*Xs)[kCols + 1] = reinterpret_cast<double (*)[kCols + 1]>(smem_raw);
    if (plasma_failed(st)) return;
    const int m = blockIdx.x, n = blockIdx.y, c0 = blockIdx.z * kCols;
    const int cols = min(kCols, plasma_tile_nview(B, n) - c0);
    if (cols <= 0) return;
    const int rows = plasma_tile_mview(B, m);
    const int col0 = n * B.nb + c0;        // global column index of chunk

    double acc[kCols];
#pragma unroll
    for (int j = 0; j < kCols; j++) acc[j] = 0.0;
    double xmax[kCols];
#pragma unroll
    for (int j = 0; j < kCols; j++) xmax[j] = 0.0;

    const int i = threadIdx.x;
    for (int k = 0; k < X.mt; k++) {
        const int kr = plasma_tile_mview(X, k);
        const double *x = (const double *)plasma_tile_addr(X, k, n);
        const int ldx = plasma_tile_mmain(X, k);
        __syncthreads();
        for (int e = threadIdx.x; e < kr * kCols; e += kResThreads) {
            int r = e % kr, c = e / kr;
            Xs[r][c] = c < cols ? x[(size_t)(c0 + c) * ldx + r] : 0.0;
        }
        __syncthreads();
        if (i < rows) {
            for (int c = 0; c < kr; c++) {
                double a = sym_at(A, uplo, m, k, i, c);
#pragma unroll
                for (int j = 0; j < kCols; j++) acc[j] += a * Xs[c][j];
            }
            if (k == m) {
#pragma unroll
                for (int j = 0; j < kCols; j++)
                    xmax[j] = fmax(xmax[j], fabs(Xs[i][j]));
            }
        }
    }
    const double *b = (const double *)plasma_tile_addr(B, m, n);
    double *r = (double *)plasma_tile_addr(R, m, n);
    const int ldb = plasma_tile_mmain(B, m), ldr = plasma_tile_mmain(R, m);
    double rmax[kCols];
#pragma unroll
    for (int j = 0; j < kCols; j++) rmax[j] = 0.0;
    if (i < rows) {
        for (int j = 0; j < cols; j++) {
            double v = b[(size_t)(c0 + j) * ldb + i] - acc[j];
            r[(size_t)(c0 + j) * ldr + i] = v;
            rmax[j] = fabs(v);
        }
    }
#pragma unroll
    for (int j = 0; j < kCols; j++) {
        double xv = xmax[j], rv = rmax[j];
        for (int off = 16; off > 0; off >>= 1) {
            xv = fmax(xv, __shfl_xor_sync(0xffffffffu, xv, off));
            rv = fmax(rv, __shfl_xor_sync(0xffffffffu, rv, off));
        }
        if ((threadIdx.x & 31) == 0 && j < cols) {
            atomic_max_nonneg(&xnorm[col0 + j], xv);
            atomic_max_nonneg(&rnorm[col0 + j], rv);
        }
    }
}

}  // namespace

extern "C" void plasma_cuda_lansy_inf(cudaStream_t s, plasma_devstat_t *st,
                                      plasma_enum_t uplo, plasma_desc_t A,
                                      double *dnorm, double *work)
{
    /* with a workspace: one pass over the stored tiles (symv.cu) */
    if (work != nullptr && plasma_cuda_lansy_tiles(s, st, uplo, A, dnorm, work))
        return;
    cudaMemsetAsync(dnorm, 0, sizeof(double), s);
    if (A.mt == 0) return;
    PLASMA_COUNT_LAUNCH();
    k_lansy_inf<<<A.mt, kThreads, 0, s>>>(A, uplo, dnorm, st);
}

extern "C" void plasma_cuda_residual(cudaStream_t s, plasma_devstat_t *st,
                                     plasma_enum_t uplo, plasma_desc_t A,
                                     plasma_desc_t B, plasma_desc_t X,
                                     plasma_desc_t R, double *xnorm,
                                     double *rnorm)
{
    cudaMemsetAsync(xnorm, 0, sizeof(double) * (size_t)B.n, s);
    cudaMemsetAsync(rnorm, 0, sizeof(double) * (size_t)B.n, s);
    if (B.mt == 0 || B.nt == 0) return;
    PLASMA_COUNT_LAUNCH();
    static unsigned long long attr_set = 0;
    if (plasma_first_on_device(&attr_set)) {
        cudaFuncSetAttribute(k_residual,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    }
    size_t smem = (size_t)X.mb * (kCols + 1) * sizeof(double);
    dim3 grid(B.mt, B.nt, ceil_div(B.nb, kCols));
    int prof = plasma_prof_begin(s);
    k_residual<<<grid, kResThreads, smem, s>>>(A, uplo, B, X, R, xnorm, rnorm, st);
    double n = B.m, nrhs = B.n;
    plasma_prof_end(prof, s, PLASMA_KCLASS_AUX, 2.0 * n * n * nrhs,
                    8.0 * (n * n / 2.0 + 3.0 * n * nrhs));
}
