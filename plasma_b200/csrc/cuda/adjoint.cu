// adjoint.cu -- reverse-mode (adjoint) kernels of the tile Cholesky factor
// and solve.  No reference counterpart: PLASMA has no derivatives; these
// serve the differentiation entry points of include/plasma_b200.h.
//
// With A = L L^T and a cotangent Lbar of L (lower triangular), the cotangent
// of the symmetric A is
//     Abar = sym(L^-T Phi(L^T Lbar) L^-1),   Phi(X) = tril(X), diagonal halved,
// and for X = A^-1 B with cotangent Xbar:
//     Bbar = A^-1 Xbar,   Lbar -= tril((Bbar X^T + X Bbar^T) L).
// The host side (compute/adjoint.c) builds both from tile steps:
//   * k_gemm_view: C = beta C + alpha op(A) op(B) on views of tile
//     descriptors -- element offsets, transpose, a triangular mask on each
//     operand (entries outside it read as zero) and on the output (entries
//     outside it are left alone or zeroed).  DMMA (mma.sync f64) for FP64,
//     the three-product TF32 split for FP32 (FP32-accurate products).  The
//     K range of a CTA is clipped to where both masked operands can be
//     non-zero, so triangular products cost what they should.
//   * k_copy_view (transposes, Phi), k_symmetrize: O(n^2) tile-layout helpers.
// The triangular solves with n right-hand sides are the library's tile
// sweeps (solve.cu).
#include "common.cuh"
#include "mma.cuh"

namespace {

constexpr int GM = 64, GN = 64, GK = 16;
constexpr int GTHREADS = 128;      // 4 warps, 32 x 32 each

typedef plasma_view_t View;

// op(V)(i, k), zero outside the triangular mask
template <typename T>
__device__ __forceinline__ const T *view_ptr(const View &v, int i, int k, bool &zero,
                                             bool &half)
{
    const int r = v.trans ? k : i, c = v.trans ? i : k;
    zero = (v.tri == 1 && r < c) || (v.tri == 2 && r > c);
    half = v.diag_scale && r == c;
    const int gr = v.r0 + r, gc = v.c0 + c;
    const int tm = gr / v.D.mb, tn = gc / v.D.nb;
    const T *t = (const T *)plasma_tile_addr(v.D, tm, tn);
    return t + (size_t)(gc - tn * v.D.nb) * plasma_tile_mmain(v.D, tm) + (gr - tm * v.D.mb);
}

template <typename T>
__device__ __forceinline__ T *out_ptr(const View &v, int i, int j)
{
    const int gr = v.r0 + i, gc = v.c0 + j;
    const int tm = gr / v.D.mb, tn = gc / v.D.nb;
    T *t = (T *)plasma_tile_addr(v.D, tm, tn);
    return t + (size_t)(gc - tn * v.D.nb) * plasma_tile_mmain(v.D, tm) + (gr - tm * v.D.mb);
}

// A block of op(V) at (i0, k0) spanning si x sk elements: when it lies in one
// storage tile, element (ii, kk) is base[ii * di + kk * dk] (returns true).
template <typename T>
__device__ __forceinline__ bool block_base(const View &v, int i0, int k0, int si, int sk,
                                           const T *&base, int &di, int &dk)
{
    // block of D: rows [r, r + sr), columns [c, c + sc)
    const int r = v.r0 + (v.trans ? k0 : i0), c = v.c0 + (v.trans ? i0 : k0);
    const int sr = v.trans ? sk : si, sc = v.trans ? si : sk;
    const int tm = r / v.D.mb, tn = c / v.D.nb;
    const int rr = r - tm * v.D.mb, cc = c - tn * v.D.nb;
    if (rr + sr > v.D.mb || cc + sc > v.D.nb) return false;
    const int ld = plasma_tile_mmain(v.D, tm);
    base = (const T *)plasma_tile_addr(v.D, tm, tn) + (size_t)cc * ld + rr;
    di = v.trans ? ld : 1;
    dk = v.trans ? 1 : ld;
    return true;
}

// K range [kb, ke) in which op(A)(i, k) op(B)(k, j) can be non-zero for
// i in [i0, i1), j in [j0, j1)
__device__ __forceinline__ void k_range(const View &a, const View &b, int K, int i0,
                                        int i1, int j0, int j1, int &kb, int &ke)
{
    kb = 0;
    ke = K;
    // op(A)(i,k): untransposed lower -> k <= i; transposed lower -> k >= i
    if (a.tri == 1) { if (a.trans) kb = max(kb, i0); else ke = min(ke, i1); }
    if (a.tri == 2) { if (a.trans) ke = min(ke, i1); else kb = max(kb, i0); }
    // op(B)(k,j): untransposed lower -> k >= j; transposed lower -> k <= j
    if (b.tri == 1) { if (b.trans) ke = min(ke, j1); else kb = max(kb, j0); }
    if (b.tri == 2) { if (b.trans) kb = max(kb, j0); else ke = min(ke, j1); }
    kb = (kb / GK) * GK;
}

template <typename T, int SPLIT>
__global__ void __launch_bounds__(GTHREADS)
k_gemm_view(int M, int N, int K, T alpha, View A, View B, T beta, View C,
            int ctri, int czero, const plasma_devstat_t *st)
{
    constexpr int LDS = GM + Pad<T>::v;
    __shared__ __align__(16) T As[2][GK][LDS];
    __shared__ __align__(16) T Bs[2][GK][LDS];
    if (plasma_failed(st)) return;
    const int i0 = blockIdx.y * GM, j0 = blockIdx.x * GN;
    const int i1 = min(M, i0 + GM), j1 = min(N, j0 + GN);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    // output block entirely outside the output mask
    const bool all_out = (ctri == 1 && j0 > i1 - 1) || (ctri == 2 && i0 > j1 - 1);
    T acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][b][c] = T(0);

    int kb, ke;
    k_range(A, B, K, i0, i1, j0, j1, kb, ke);
    if (all_out) ke = kb;
    // masks in the coordinates of the untransposed view
    auto masked = [](const View &v, int i, int k) {
        const int r = v.trans ? k : i, c = v.trans ? i : k;
        return (v.tri == 1 && r < c) || (v.tri == 2 && r > c);
    };
    auto halved = [](const View &v, int i, int k) { return v.diag_scale && i == k; };
    auto stage = [&](int k0, int buf) {
        const T *ba, *bb;
        int dia, dka, dib, dkb;
        const bool fa = block_base<T>(A, i0, k0, GM, GK, ba, dia, dka);
        // op(B)(k, j): first index k, second j
        const bool fb = block_base<T>(B, k0, j0, GK, GN, bb, dib, dkb);
        for (int e = tid; e < GK * GM; e += GTHREADS) {
            const int ii = e % GM, kk = e / GM;
            const int i = i0 + ii, k = k0 + kk;
            const bool in = i < M && k < ke && !masked(A, i, k);
            const T *p = (const T *)A.D.matrix;
            if (in) {
                if (fa) {
                    p = ba + (size_t)ii * dia + (size_t)kk * dka;
                } else {
                    bool z, h;
                    p = view_ptr<T>(A, i, k, z, h);
                }
            }
            if (in && halved(A, i, k)) As[buf][kk][ii] = T(0.5) * *p;
            else cp_async_el(&As[buf][kk][ii], p, in);
        }
        for (int e = tid; e < GK * GN; e += GTHREADS) {
            const int jj = e % GN, kk = e / GN;
            const int j = j0 + jj, k = k0 + kk;
            // op(B)(k, j): the view's "row" index is k
            const bool in = j < N && k < ke && !masked(B, k, j);
            const T *p = (const T *)B.D.matrix;
            if (in) {
                if (fb) {
                    p = bb + (size_t)kk * dib + (size_t)jj * dkb;
                } else {
                    bool z, h;
                    p = view_ptr<T>(B, k, j, z, h);
                }
            }
            if (in && halved(B, k, j)) Bs[buf][kk][jj] = T(0.5) * *p;
            else cp_async_el(&Bs[buf][kk][jj], p, in);
        }
        cp_async_commit();
    };
    if (kb < ke) {
        stage(kb, 0);
        int buf = 0;
        for (int k0 = kb; k0 < ke; k0 += GK, buf ^= 1) {
            if (k0 + GK < ke) {
                stage(k0 + GK, buf ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
#pragma unroll
            for (int k8 = 0; k8 < GK; k8 += 8) {
                T bf[4][2];
#pragma unroll
                for (int ni = 0; ni < 4; ni++) {
                    bf[ni][0] = Bs[buf][k8 + t][wn + ni * 8 + g];
                    bf[ni][1] = Bs[buf][k8 + t + 4][wn + ni * 8 + g];
                }
#pragma unroll
                for (int mi = 0; mi < 2; mi++) {
                    T af[4];
                    af[0] = As[buf][k8 + t][wm + mi * 16 + g];
                    af[1] = As[buf][k8 + t][wm + mi * 16 + g + 8];
                    af[2] = As[buf][k8 + t + 4][wm + mi * 16 + g];
                    af[3] = As[buf][k8 + t + 4][wm + mi * 16 + g + 8];
#pragma unroll
                    for (int ni = 0; ni < 4; ni++) mma8<SPLIT>(acc[mi][ni], af, bf[ni]);
                }
            }
            __syncthreads();
        }
    }
    // epilogue
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int i = i0 + wm + mi * 16 + g + 8 * h;
                    const int j = j0 + wn + ni * 8 + 2 * t + e;
                    if (i >= M || j >= N) continue;
                    const bool in = ctri == 0 || (ctri == 1 && i >= j) || (ctri == 2 && i <= j);
                    T *p = out_ptr<T>(C, i, j);
                    if (!in) {
                        if (czero) *p = T(0);
                        continue;
                    }
                    const T v = alpha * acc[mi][ni][2 * h + e];
                    *p = beta == T(0) ? v : beta * *p + v;
                }
}

// dst(i,j) = op(src)(i,j), 32 x 32 blocks staged in shared memory so that
// both the read of src (in its own orientation) and the write are along
// tile columns.
template <typename T>
__global__ void __launch_bounds__(256)
k_copy_view(int M, int N, View src, View dst, const plasma_devstat_t *st)
{
    __shared__ T blk[32][33];
    if (plasma_failed(st)) return;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 8 rows of 32
    // read: the element index along tile columns of src is the row of the
    // untransposed view
    for (int q = ty; q < 32; q += 8) {
        // untransposed: (i, j) = (i0 + tx, j0 + q); transposed: (i0 + q, j0 + tx)
        const int i = src.trans ? i0 + q : i0 + tx;
        const int j = src.trans ? j0 + tx : j0 + q;
        T v = T(0);
        if (i < M && j < N) {
            bool zero, half;
            const T *p = view_ptr<T>(src, i, j, zero, half);
            v = zero ? T(0) : (half ? T(0.5) * *p : *p);
        }
        if (src.trans) blk[q][tx] = v; else blk[tx][q] = v;
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        const int i = i0 + tx, j = j0 + q;
        if (i < M && j < N) *out_ptr<T>(dst, i, j) = blk[tx][q];
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_symmetrize(int n, View src, View dst, const plasma_devstat_t *st)
{
    __shared__ T a[32][33], b[32][33];
    if (plasma_failed(st)) return;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int q = ty; q < 32; q += 8) {
        bool zero, half;
        // a(i, j) = src(i0 + tx, j0 + q); b holds src(j0 + tx, i0 + q)
        a[tx][q] = (i0 + tx < n && j0 + q < n) ? *view_ptr<T>(src, i0 + tx, j0 + q, zero, half) : T(0);
        b[tx][q] = (j0 + tx < n && i0 + q < n) ? *view_ptr<T>(src, j0 + tx, i0 + q, zero, half) : T(0);
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        const int i = i0 + tx, j = j0 + q;
        // src(j, i) = b[q][tx]
        if (i < n && j < n) *out_ptr<T>(dst, i, j) = T(0.5) * (a[tx][q] + b[q][tx]);
    }
}

}  // namespace

extern "C" void plasma_cuda_gemm_view(cudaStream_t s, plasma_devstat_t *st, int M, int N,
                                      int K, double alpha, plasma_view_t A, plasma_view_t B,
                                      double beta, plasma_view_t C, int ctri, int czero)
{
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    if (C.D.precision == PlasmaRealDouble)
        k_gemm_view<double, 1><<<grid, GTHREADS, 0, s>>>(M, N, K, alpha, A, B, beta, C,
                                                          ctri, czero, st);
    else
        k_gemm_view<float, 3><<<grid, GTHREADS, 0, s>>>(M, N, K, (float)alpha, A, B,
                                                         (float)beta, C, ctri, czero, st);
    plasma_prof_end(prof, s, PLASMA_KCLASS_UPDATE, 2.0 * M * N * (double)K, 0.0);
}

extern "C" void plasma_cuda_copy_view(cudaStream_t s, plasma_devstat_t *st, int M, int N,
                                      plasma_view_t src, plasma_view_t dst)
{
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + 31) / 32, (M + 31) / 32);
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    if (dst.D.precision == PlasmaRealDouble)
        k_copy_view<double><<<grid, 256, 0, s>>>(M, N, src, dst, st);
    else
        k_copy_view<float><<<grid, 256, 0, s>>>(M, N, src, dst, st);
    plasma_prof_end(prof, s, PLASMA_KCLASS_AUX, 0.0,
                    2.0 * M * N * plasma_element_size(dst.D.precision));
}

extern "C" void plasma_cuda_symmetrize(cudaStream_t s, plasma_devstat_t *st, int n,
                                       plasma_view_t src, plasma_view_t dst)
{
    if (n <= 0) return;
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    if (dst.D.precision == PlasmaRealDouble)
        k_symmetrize<double><<<grid, 256, 0, s>>>(n, src, dst, st);
    else
        k_symmetrize<float><<<grid, 256, 0, s>>>(n, src, dst, st);
    plasma_prof_end(prof, s, PLASMA_KCLASS_AUX, 0.0,
                    3.0 * (double)n * n * plasma_element_size(dst.D.precision));
}
