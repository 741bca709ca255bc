// vec.cu -- vector kernels of the refinement loops (FP64 working precision):
// block dot products with a deterministic two-stage reduction, the classical
// Gram-Schmidt step of GMRES, scaled copies, FP64 <-> FP32 conversion and the
// transfer of one column of a tile descriptor to a contiguous vector.
#include "common.cuh"

namespace {

constexpr int VT = 256;
constexpr int VBLOCKS = 296;   // two CTAs per SM

// partial[i * VBLOCKS + b] = sum over the block's range of V[i][e] * w[e]
__global__ void __launch_bounds__(VT)
k_dots(const double *V, size_t ldv, int nv, const double *w, size_t n, double *partial)
{
    __shared__ double red[VT / 32];
    const int i = blockIdx.y;
    const double *v = V + (size_t)i * ldv;
    double s = 0.0;
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < n; e += (size_t)gridDim.x * VT)
        s += v[e] * w[e];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < VT / 32; k++) t += red[k];
        partial[(size_t)i * gridDim.x + blockIdx.x] = t;
    }
}

// out[i] = sum_b partial[i * nb + b]  (fixed order)
__global__ void k_dots_final(const double *partial, int nblk, int nv, double *out)
{
    int i = threadIdx.x;
    if (i >= nv) return;
    double t = 0.0;
    for (int b = 0; b < nblk; b++) t += partial[(size_t)i * nblk + b];
    out[i] = t;
}

// w -= sum_i h[i] V[i]
__global__ void __launch_bounds__(VT)
k_sub_combo(const double *V, size_t ldv, int nv, const double *h, double *w, size_t n)
{
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < n; e += (size_t)gridDim.x * VT) {
        double s = 0.0;
        for (int i = 0; i < nv; i++) s += h[i] * V[(size_t)i * ldv + e];
        w[e] -= s;
    }
}

// y = alpha * x (+ y when accumulate)
__global__ void __launch_bounds__(VT)
k_axpby(double alpha, const double *x, double *y, size_t n, int accumulate)
{
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < n; e += (size_t)gridDim.x * VT)
        y[e] = alpha * x[e] + (accumulate ? y[e] : 0.0);
}

// y = sum_i c[i] V[i] (+ y)
__global__ void __launch_bounds__(VT)
k_combo(const double *V, size_t ldv, int nv, const double *c, double *y, size_t n,
        int accumulate)
{
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < n; e += (size_t)gridDim.x * VT) {
        double s = 0.0;
        for (int i = 0; i < nv; i++) s += c[i] * V[(size_t)i * ldv + e];
        y[e] = s + (accumulate ? y[e] : 0.0);
    }
}

// FP64 -> FP32 (zero beyond n up to npad), optionally scaled by s[e];
// flags FP32 overflow like dlag2s
__global__ void __launch_bounds__(VT)
k_d2s(const double *x, const double *sc, float *y, size_t n, size_t npad,
      plasma_devstat_t *st, int call)
{
    bool ovf = false;
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < npad; e += (size_t)gridDim.x * VT) {
        double v = e < n ? x[e] * (sc ? sc[e] : 1.0) : 0.0;
        if (v > 3.4028234663852886e38 || v < -3.4028234663852886e38) ovf = true;
        y[e] = (float)v;
    }
    if (ovf) plasma_fail(st, 1, call);
}

__global__ void __launch_bounds__(VT)
k_s2d(const float *x, const double *sc, double *y, size_t n)
{
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < n; e += (size_t)gridDim.x * VT)
        y[e] = (double)x[e] * (sc ? sc[e] : 1.0);
}

// d[i] = 1 / sqrt(A(i,i)) for i < n (A FP64, any storage), 1 beyond
__global__ void __launch_bounds__(VT)
k_diag_rsqrt(plasma_desc_t A, double *d, size_t n, size_t npad)
{
    for (size_t e = (size_t)blockIdx.x * VT + threadIdx.x; e < npad; e += (size_t)gridDim.x * VT) {
        double v = 1.0;
        if (e < n) {
            int m = (int)(e / A.mb), r = (int)(e % A.mb);
            const double *t = (const double *)plasma_tile_addr(A, m, m);
            double a = t[(size_t)r * plasma_tile_mmain(A, m) + r];
            v = a > 0.0 ? 1.0 / sqrt(a) : 1.0;
        }
        d[e] = v;
    }
}

// As(i,j) <- d_i As(i,j) d_j on the stored triangle tiles, then the diagonal
// gets + shift (FP32 factor operand; d FP64 of length npad)
__global__ void __launch_bounds__(VT)
k_scale_shift(plasma_desc_t As, int uplo, const double *d, float shift)
{
    const int m = blockIdx.x, n = blockIdx.y;
    if (uplo == PlasmaLower ? n > m : n < m) return;
    float *t = (float *)plasma_tile_addr(As, m, n);
    const int ld = plasma_tile_mmain(As, m);
    const int rows = plasma_tile_mview(As, m), cols = plasma_tile_nview(As, n);
    for (int e = threadIdx.x; e < rows * cols; e += VT) {
        int r = e % rows, c = e / rows;
        int gi = m * As.mb + r, gj = n * As.nb + c;
        double v = (double)t[(size_t)c * ld + r] * d[gi] * d[gj];
        if (gi == gj) v += shift;
        t[(size_t)c * ld + r] = (float)v;
    }
}

// column j of a tile descriptor <-> contiguous vector
template <typename T, bool TO_VEC>
__global__ void __launch_bounds__(VT)
k_column(plasma_desc_t D, int j, T *v)
{
    const int n = D.m;
    const int jt = j / D.nb, jj = j % D.nb;
    for (int e = blockIdx.x * VT + threadIdx.x; e < n; e += gridDim.x * VT) {
        int m = e / D.mb, r = e % D.mb;
        T *t = (T *)plasma_tile_addr(D, m, jt);
        T *p = t + (size_t)jj * plasma_tile_mmain(D, m) + r;
        if (TO_VEC) v[e] = *p;
        else *p = v[e];
    }
}

unsigned blocks_for(size_t n)
{
    size_t b = (n + VT - 1) / VT;
    return (unsigned)(b < VBLOCKS ? (b ? b : 1) : VBLOCKS);
}

}  // namespace

extern "C" size_t plasma_cuda_dots_work(int nv)
{
    return sizeof(double) * (size_t)nv * VBLOCKS;
}

// out[i] = V_i . w for i < nv (V_i = V + i*ldv); deterministic
extern "C" void plasma_cuda_dots(cudaStream_t s, const double *V, size_t ldv, int nv,
                                 const double *w, size_t n, double *out, double *work)
{
    unsigned nb = blocks_for(n);
    PLASMA_COUNT_LAUNCH();
    k_dots<<<dim3(nb, nv), VT, 0, s>>>(V, ldv, nv, w, n, work);
    PLASMA_COUNT_LAUNCH();
    k_dots_final<<<1, 1024, 0, s>>>(work, (int)nb, nv, out);
}

extern "C" void plasma_cuda_sub_combo(cudaStream_t s, const double *V, size_t ldv,
                                      int nv, const double *h, double *w, size_t n)
{
    PLASMA_COUNT_LAUNCH();
    k_sub_combo<<<blocks_for(n), VT, 0, s>>>(V, ldv, nv, h, w, n);
}

extern "C" void plasma_cuda_axpby(cudaStream_t s, double alpha, const double *x,
                                  double *y, size_t n, int accumulate)
{
    PLASMA_COUNT_LAUNCH();
    k_axpby<<<blocks_for(n), VT, 0, s>>>(alpha, x, y, n, accumulate);
}

extern "C" void plasma_cuda_combo(cudaStream_t s, const double *V, size_t ldv, int nv,
                                  const double *c, double *y, size_t n, int accumulate)
{
    PLASMA_COUNT_LAUNCH();
    k_combo<<<blocks_for(n), VT, 0, s>>>(V, ldv, nv, c, y, n, accumulate);
}

extern "C" void plasma_cuda_d2s(cudaStream_t s, const double *x, const double *sc,
                                float *y, size_t n, size_t npad, plasma_devstat_t *st,
                                int call)
{
    PLASMA_COUNT_LAUNCH();
    k_d2s<<<blocks_for(npad), VT, 0, s>>>(x, sc, y, n, npad, st, call);
}

extern "C" void plasma_cuda_s2d(cudaStream_t s, const float *x, const double *sc,
                                double *y, size_t n)
{
    PLASMA_COUNT_LAUNCH();
    k_s2d<<<blocks_for(n), VT, 0, s>>>(x, sc, y, n);
}

extern "C" void plasma_cuda_diag_rsqrt(cudaStream_t s, plasma_desc_t A, double *d,
                                       size_t n, size_t npad)
{
    PLASMA_COUNT_LAUNCH();
    k_diag_rsqrt<<<blocks_for(npad), VT, 0, s>>>(A, d, n, npad);
}

extern "C" void plasma_cuda_scale_shift(cudaStream_t s, plasma_desc_t As, int uplo,
                                        const double *d, float shift)
{
    PLASMA_COUNT_LAUNCH();
    k_scale_shift<<<dim3(As.mt, As.nt), VT, 0, s>>>(As, uplo, d, shift);
}

extern "C" void plasma_cuda_column(cudaStream_t s, plasma_desc_t D, int j, void *v,
                                   int to_vec)
{
    PLASMA_COUNT_LAUNCH();
    unsigned nb = blocks_for((size_t)D.m);
    if (D.precision == PlasmaRealDouble) {
        if (to_vec) k_column<double, true><<<nb, VT, 0, s>>>(D, j, (double *)v);
        else        k_column<double, false><<<nb, VT, 0, s>>>(D, j, (double *)v);
    } else {
        if (to_vec) k_column<float, true><<<nb, VT, 0, s>>>(D, j, (float *)v);
        else        k_column<float, false><<<nb, VT, 0, s>>>(D, j, (float *)v);
    }
}
