// panel.cu -- FP64 critical path of a Cholesky step on the tensor cores:
// the diagonal-tile factorisation and the panel triangular solve
// (compute/pzpotrf.c:41-56: plasma_core_dpotrf on A(k,k), then
// plasma_core_dtrsm(Right, Lower, Trans, NonUnit) on every A(m,k), m > k).
//
// k_potrf_diag_dmma -- one CTA factors the diagonal tile left-looking in
//   64-column panels.  The update of a panel by the columns to its left,
//   P -= L(j0:n, 0:j0) L(j0:j0+64, 0:j0)^T, runs on DMMA (mma.sync f64); the
//   64-wide panel is then factored in shared memory as four 16-column
//   sub-panels: DMMA update by the sub-panels to its left, one warp factors
//   the 16x16 diagonal block through shuffles, and every thread solves one
//   row below it (three barriers per 16 columns).
//   Pivot test and info as LAPACK dpotrf (first pivot not > 0, or NaN).
// k_trsm_panel_dmma -- X L^T = A(m,k) for all m > k.  A CTA keeps 64 rows of
//   one tile (all nb columns) in shared memory and walks the 64-column blocks
//   left to right:  Y_j = X_j - X_{<j} L_{j,<j}^T  (DMMA, L streamed from L2
//   through a cp.async double buffer), then X_j L_jj^T = Y_j by right-looking
//   substitution, four lanes per row exchanging the solved entry by shuffle.
#include "common.cuh"
#include "mma.cuh"

namespace {

constexpr int PB = 64;          // panel / block width
constexpr int NBMAX = 256;      // largest tile handled here
constexpr int THR = 256;

// ------------------------------------------------------------------------
// diagonal tile
// ------------------------------------------------------------------------
constexpr int DKC = 16;             // K chunk of the left-looking update
constexpr int SP = 16;              // sub-panel width inside a panel
template <typename T> constexpr int diag_smem()
{
    return (PB * (NBMAX + Pad<T>::v) + 2 * DKC * (NBMAX + Pad<T>::v) +
            2 * DKC * (PB + Pad<T>::v)) * (int)sizeof(T);
}

template <typename T, int SPLIT>
__global__ void __launch_bounds__(THR, 1)
k_potrf_diag_mma(plasma_desc_t A, int k, int iinfo, plasma_devstat_t *st,
                 int call)
{
    constexpr int P_LD = NBMAX + Pad<T>::v;   // panel stored [col][row]
    constexpr int SA_LD = NBMAX + Pad<T>::v;  // staged L rows chunk [k][row]
    constexpr int SB_LD = PB + Pad<T>::v;     // staged L panel rows chunk
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *P = reinterpret_cast<T *>(smem_raw);                 // [PB][P_LD]
    T *Sa = P + PB * P_LD;                                  // [2][DKC][SA_LD]
    T *Sb = Sa + 2 * DKC * SA_LD;                           // [2][DKC][SB_LD]
    if (plasma_failed(st)) return;
    T *L = (T *)plasma_tile_addr(A, k, k);
    const int ld = plasma_tile_mmain(A, k);
    const int n = plasma_tile_mview(A, k);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    for (int j0 = 0; j0 < n; j0 += PB) {
        const int jb = min(PB, n - j0);
        const int R = n - j0;
        __syncthreads();
        // ---- load the panel P[c][r] = L(j0+r, j0+c) (lower part), async
        for (int e = tid; e < R * PB; e += THR) {
            int r = e % R, c = e / R;
            bool v = c < jb && r >= c;
            cp_async_el(P + c * P_LD + r, v ? L + (size_t)(j0 + c) * ld + j0 + r : L, v);
        }
        cp_async_commit();
        // ---- left-looking update on DMMA: warp w owns rows 32w..32w+31,
        //      operand chunks double-buffered through cp.async
        if (j0 > 0) {
            T acc[2][8][4];
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 8; b++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[a][b][c] = T(0);
            auto stage = [&](int kc, int buf) {
                T *sa = Sa + buf * DKC * SA_LD;
                T *sb = Sb + buf * DKC * SB_LD;
                for (int e = tid; e < DKC * NBMAX; e += THR) {
                    int r = e % NBMAX, kk = e / NBMAX;
                    bool v = r < R;
                    cp_async_el(sa + kk * SA_LD + r,
                               v ? L + (size_t)(kc + kk) * ld + j0 + r : L, v);
                }
                for (int e = tid; e < DKC * PB; e += THR) {
                    int c = e % PB, kk = e / PB;
                    bool v = c < jb;
                    cp_async_el(sb + kk * SB_LD + c,
                               v ? L + (size_t)(kc + kk) * ld + j0 + c : L, v);
                }
                cp_async_commit();
            };
            const int nkc = j0 / DKC;
            stage(0, 0);
            for (int q = 0; q < nkc; q++) {
                if (q + 1 < nkc) {
                    stage((q + 1) * DKC, (q + 1) & 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                const T *sa = Sa + (q & 1) * DKC * SA_LD;
                const T *sb = Sb + (q & 1) * DKC * SB_LD;
                if (warp * 32 < R) {
#pragma unroll
                    for (int k8 = 0; k8 < DKC; k8 += 8) {
                        T bf[8][2];
#pragma unroll
                        for (int ni = 0; ni < 8; ni++) {
                            bf[ni][0] = sb[(k8 + t) * SB_LD + ni * 8 + g];
                            bf[ni][1] = sb[(k8 + t + 4) * SB_LD + ni * 8 + g];
                        }
#pragma unroll
                        for (int mi = 0; mi < 2; mi++) {
                            const T *as = sa + warp * 32 + mi * 16;
                            T af[4];
                            af[0] = as[(k8 + t) * SA_LD + g];
                            af[1] = as[(k8 + t) * SA_LD + g + 8];
                            af[2] = as[(k8 + t + 4) * SA_LD + g];
                            af[3] = as[(k8 + t + 4) * SA_LD + g + 8];
#pragma unroll
                            for (int ni = 0; ni < 8; ni++)
                                mma8<SPLIT>(acc[mi][ni], af, bf[ni]);
                        }
                    }
                }
                __syncthreads();
            }
            cp_async_wait<0>();
            __syncthreads();
            if (warp * 32 < R) {
#pragma unroll
                for (int mi = 0; mi < 2; mi++)
#pragma unroll
                    for (int ni = 0; ni < 8; ni++)
#pragma unroll
                        for (int h = 0; h < 2; h++)
#pragma unroll
                            for (int e = 0; e < 2; e++) {
                                int r = warp * 32 + mi * 16 + g + 8 * h;
                                int c = ni * 8 + 2 * t + e;
                                if (r < R && c < jb && r >= c)
                                    P[c * P_LD + r] -= acc[mi][ni][2 * h + e];
                            }
            }
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        // ---- factor the panel in 16-column sub-panels (all in shared memory)
        int *flag_s = reinterpret_cast<int *>(Sa);
        T *rdiag_s = Sa + 4;               // reciprocals of the block diagonal
        for (int cs = 0; cs < jb; cs += SP) {
            const int sw = min(SP, jb - cs);
            // (a) sub-panel -= previous sub-panels of this panel (DMMA, K = cs)
            if (cs > 0) {
                T acc[2][2][4];
#pragma unroll
                for (int a = 0; a < 2; a++)
#pragma unroll
                    for (int b = 0; b < 2; b++)
#pragma unroll
                        for (int c = 0; c < 4; c++) acc[a][b][c] = T(0);
                const int rbase = warp * 32;      // rows of this warp (panel-relative)
                if (rbase + 31 >= cs && rbase < R) {
                    for (int k8 = 0; k8 < cs; k8 += 8) {
                        T bf[2][2];
#pragma unroll
                        for (int ni = 0; ni < 2; ni++) {
                            bf[ni][0] = P[(k8 + t) * P_LD + cs + ni * 8 + g];
                            bf[ni][1] = P[(k8 + t + 4) * P_LD + cs + ni * 8 + g];
                        }
#pragma unroll
                        for (int mi = 0; mi < 2; mi++) {
                            const T *as = P + rbase + mi * 16;
                            T af[4];
                            af[0] = as[(k8 + t) * P_LD + g];
                            af[1] = as[(k8 + t) * P_LD + g + 8];
                            af[2] = as[(k8 + t + 4) * P_LD + g];
                            af[3] = as[(k8 + t + 4) * P_LD + g + 8];
#pragma unroll
                            for (int ni = 0; ni < 2; ni++)
                                mma8<SPLIT>(acc[mi][ni], af, bf[ni]);
                        }
                    }
                }
                __syncthreads();
                if (rbase + 31 >= cs && rbase < R) {
#pragma unroll
                    for (int mi = 0; mi < 2; mi++)
#pragma unroll
                        for (int ni = 0; ni < 2; ni++)
#pragma unroll
                            for (int h = 0; h < 2; h++)
#pragma unroll
                                for (int e = 0; e < 2; e++) {
                                    int r = rbase + mi * 16 + g + 8 * h;
                                    int c = cs + ni * 8 + 2 * t + e;
                                    if (r < R && c < cs + sw && r >= c)
                                        P[c * P_LD + r] -= acc[mi][ni][2 * h + e];
                                }
                }
                __syncthreads();
            }
            // (b) 16x16 diagonal block: one warp, lane i < sw owns row i
            if (warp == 0) {
                T v[SP];
#pragma unroll
                for (int c = 0; c < SP; c++)
                    v[c] = (lane < sw && c < sw && lane >= c) ? P[(cs + c) * P_LD + cs + lane] : T(0);
                int bad = 0;
#pragma unroll
                for (int c = 0; c < SP; c++) {
                    if (c < sw) {
                        T d = __shfl_sync(0xffffffffu, v[c], c);
                        bool ok = d > T(0);
                        if (!ok && bad == 0) bad = c + 1;
                        T sd = ok ? sqrt(d) : T(1);
                        T rd = T(1) / sd;
                        if (lane >= c) v[c] = (lane == c) ? sd : v[c] * rd;
#pragma unroll
                        for (int c2 = c + 1; c2 < SP; c2++) {
                            T lc2 = __shfl_sync(0xffffffffu, v[c], c2);
                            if (c2 < sw && lane >= c2) v[c2] -= v[c] * lc2;
                        }
                    }
                }
                if (lane < sw) {
#pragma unroll
                    for (int c = 0; c < SP; c++)
                        if (c < sw && lane >= c) P[(cs + c) * P_LD + cs + lane] = v[c];
                    rdiag_s[lane] = T(1) / P[(cs + lane) * P_LD + cs + lane];
                }
                if (lane == 0) flag_s[0] = bad;
            }
            __syncthreads();
            if (flag_s[0] != 0) {
                if (tid == 0) plasma_fail(st, iinfo + j0 + cs + flag_s[0], call);
                return;
            }
            // (c) rows below the block: x L_blk^T = p, one thread per row
            {
                const int r = cs + sw + tid;
                if (r < R) {
                    T x[SP];
#pragma unroll
                    for (int c = 0; c < SP; c++)
                        x[c] = c < sw ? P[(cs + c) * P_LD + r] : T(0);
#pragma unroll
                    for (int c = 0; c < SP; c++) {
                        if (c < sw) {
                            x[c] = x[c] * rdiag_s[c];
#pragma unroll
                            for (int c2 = c + 1; c2 < SP; c2++)
                                if (c2 < sw) x[c2] -= x[c] * P[(cs + c) * P_LD + cs + c2];
                        }
                    }
#pragma unroll
                    for (int c = 0; c < SP; c++)
                        if (c < sw) P[(cs + c) * P_LD + r] = x[c];
                }
            }
            __syncthreads();
        }
        // ---- store the panel (lower part only)
        for (int e = tid; e < R * jb; e += THR) {
            int rr = e % R, c = e / R;
            if (rr >= c) L[(size_t)(j0 + c) * ld + j0 + rr] = P[c * P_LD + rr];
        }
    }
}

// ------------------------------------------------------------------------
// panel solve
// ------------------------------------------------------------------------
constexpr int TR = 64;               // rows per CTA
constexpr int TKC = 16;
static_assert(THR == 4 * TR, "four lanes per row in the block solve");
template <typename T> constexpr int trsm_smem()
{
    return (NBMAX * (TR + Pad<T>::v) + 2 * TKC * (PB + Pad<T>::v) +
            PB * (PB + Pad<T>::v) + PB) * (int)sizeof(T);
}

template <typename T, int SPLIT>
__global__ void __launch_bounds__(THR, 1)
k_trsm_panel_mma(plasma_desc_t A, int k, int mlo, const plasma_devstat_t *st)
{
    constexpr int X_LD = TR + Pad<T>::v;      // X stored [col][row]
    constexpr int L_LD = PB + Pad<T>::v;      // staged L chunk [k][row-of-block]
    constexpr int EPV = 16 / (int)sizeof(T);  // elements per 16-byte copy
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *X = reinterpret_cast<T *>(smem_raw);                 // [NBMAX][X_LD]
    T *Ls = X + NBMAX * X_LD;                                // [2][TKC][L_LD]
    T *Ws = Ls + 2 * TKC * L_LD;                             // L_jj [PB][L_LD]
    T *Rd = Ws + PB * L_LD;                                  // 1 / diag(L_jj)
    if (plasma_failed(st)) return;

    const int m = mlo + blockIdx.x;
    const T *Lkk = (const T *)plasma_tile_addr(A, k, k);
    const int ldl = plasma_tile_mmain(A, k);
    const int nb = plasma_tile_mview(A, k);          // multiple of 64 here
    T *B = (T *)plasma_tile_addr(A, m, k);
    const int ldb = plasma_tile_mmain(A, m);
    const int rows = plasma_tile_mview(A, m);
    const int r0 = blockIdx.y * TR;
    if (r0 >= rows) return;
    const int nr = min(TR, rows - r0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp >> 2;       // 0..1 : 32 rows
    const int wn = warp & 3;        // 0..3 : 16 cols

    for (int e = tid; e < nb * TR; e += THR) {
        int r = e % TR, c = e / TR;
        bool v = r < nr;
        cp_async_el(X + c * X_LD + r, v ? B + (size_t)c * ldb + r0 + r : B, v);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    for (int j = 0; j < nb; j += PB) {
        T acc[2][2][4];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][b][c] = T(0);
        // S = X_{<j} L_{j,<j}^T : K = j, L rows j..j+63 staged per chunk
        const int nkc = j / TKC;
        auto stage = [&](int kc, int buf) {
            T *dst = Ls + buf * TKC * L_LD;
            for (int e = tid; e < TKC * PB / EPV; e += THR) {
                int rr = EPV * (e % (PB / EPV)), kk = e / (PB / EPV);
                cp_async_16(dst + kk * L_LD + rr,
                            Lkk + (size_t)(kc + kk) * ldl + j + rr, true);
            }
            cp_async_commit();
        };
        if (nkc > 0) stage(0, 0);
        for (int q = 0; q < nkc; q++) {
            if (q + 1 < nkc) {
                stage((q + 1) * TKC, (q + 1) & 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const T *ls = Ls + (q & 1) * TKC * L_LD + wn * 16;
            const T *xs = X + (size_t)(q * TKC) * X_LD + wm * 32;
#pragma unroll
            for (int k8 = 0; k8 < TKC; k8 += 8) {
                T bf[2][2];
#pragma unroll
                for (int ni = 0; ni < 2; ni++) {
                    bf[ni][0] = ls[(k8 + t) * L_LD + ni * 8 + g];
                    bf[ni][1] = ls[(k8 + t + 4) * L_LD + ni * 8 + g];
                }
#pragma unroll
                for (int mi = 0; mi < 2; mi++) {
                    T af[4];
                    af[0] = xs[(k8 + t) * X_LD + mi * 16 + g];
                    af[1] = xs[(k8 + t) * X_LD + mi * 16 + g + 8];
                    af[2] = xs[(k8 + t + 4) * X_LD + mi * 16 + g];
                    af[3] = xs[(k8 + t + 4) * X_LD + mi * 16 + g + 8];
#pragma unroll
                    for (int ni = 0; ni < 2; ni++)
                        mma8<SPLIT>(acc[mi][ni], af, bf[ni]);
                }
            }
            __syncthreads();
        }
        // Y_j = X_j - S, written over X_j; stage L_jj (column-major, ld L_LD)
        for (int e = tid; e < PB * PB; e += THR) {
            int i = e % PB, c = e / PB;
            cp_async_el(Ws + c * L_LD + i, Lkk + (size_t)(j + c) * ldl + j + i, true);
        }
        cp_async_commit();
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int ni = 0; ni < 2; ni++)
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        int r = wm * 32 + mi * 16 + g + 8 * h;
                        int c = j + wn * 16 + ni * 8 + 2 * t + e;
                        X[c * X_LD + r] -= acc[mi][ni][2 * h + e];
                    }
        cp_async_wait<0>();
        __syncthreads();
        if (tid < PB) Rd[tid] = T(1) / Ws[tid * L_LD + tid];
        __syncthreads();
        // X_j L_jj^T = Y_j: row r = tid/4, lane q = tid%4 owns columns
        // q, q+4, ..., q+60 of the block
        {
            const int r = tid >> 2, q = tid & 3;
            T y[PB / 4];
#pragma unroll
            for (int i = 0; i < PB / 4; i++)
                y[i] = X[(size_t)(j + q + 4 * i) * X_LD + r];
#pragma unroll
            for (int c = 0; c < PB; c++) {
                T mine = y[c / 4];
                T x = __shfl_sync(0xffffffffu, mine, (lane & ~3) | (c & 3));
                x = x * Rd[c];
                if (q == (c & 3)) y[c / 4] = x;
#pragma unroll
                for (int i = 0; i < PB / 4; i++) {
                    int c2 = q + 4 * i;
                    if (c2 > c) y[i] -= x * Ws[c * L_LD + c2];
                }
            }
#pragma unroll
            for (int i = 0; i < PB / 4; i++)
                X[(size_t)(j + q + 4 * i) * X_LD + r] = y[i];
        }
        __syncthreads();
    }
    for (int e = tid; e < nb * TR; e += THR) {
        int r = e % TR, c = e / TR;
        if (r < nr) B[(size_t)c * ldb + r0 + r] = X[c * X_LD + r];
    }
}

template <typename T, int SPLIT>
void launch_diag(cudaStream_t s, plasma_devstat_t *st, int call,
                 const plasma_desc_t &A, int k, int iinfo)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_potrf_diag_mma<T, SPLIT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem<T>());
    }
    k_potrf_diag_mma<T, SPLIT><<<1, THR, diag_smem<T>(), s>>>(A, k, iinfo, st, call);
}

template <typename T, int SPLIT>
void launch_trsm(cudaStream_t s, plasma_devstat_t *st, const plasma_desc_t &A,
                 int k, int mlo, int mhi)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsm_panel_mma<T, SPLIT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, trsm_smem<T>());
    }
    dim3 grid((unsigned)(mhi - mlo), (unsigned)ceil_div(A.mb, TR));
    k_trsm_panel_mma<T, SPLIT><<<grid, THR, trsm_smem<T>(), s>>>(A, k, mlo, st);
}

// 3 = FP32-accurate split for plain FP32 factors, 1 for TF32/BF16 factors
int g_fp32_split = 3;

}  // namespace

extern "C" void plasma_cuda_panel_set_split(int split)
{
    g_fp32_split = split == 1 ? 1 : 3;
}

// Fast path: lower storage, square tiles with nb <= 256.  Returns 0 when the
// request is not eligible (the caller then uses the generic kernels).
extern "C" int plasma_cuda_potrf_diag_fast(cudaStream_t s, plasma_devstat_t *st,
                                          int call, plasma_enum_t uplo,
                                          plasma_desc_t A, int k, int iinfo)
{
    if (uplo != PlasmaLower || A.mb > NBMAX || A.mb != A.nb ||
        (A.precision != PlasmaRealDouble && A.precision != PlasmaRealFloat))
        return 0;
    PLASMA_COUNT_LAUNCH();
    double nk = plasma_tile_mview(A, k);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        launch_diag<double, 1>(s, st, call, A, k, iinfo);
    else if (plasma_cuda_potrf_diag_smem(s, st, call, uplo, A, k, iinfo, g_fp32_split))
        ;   // FP32 tile held in shared memory (potrf_smem.cu)
    else if (g_fp32_split == 1)
        launch_diag<float, 1>(s, st, call, A, k, iinfo);
    else
        launch_diag<float, 3>(s, st, call, A, k, iinfo);
    plasma_prof_end(prof, s, PLASMA_KCLASS_POTRF, nk * nk * nk / 3.0,
                    nk * nk * 2.0 * plasma_element_size(A.precision));
    return 1;
}

extern "C" int plasma_cuda_trsm_panel_fast(cudaStream_t s, plasma_devstat_t *st,
                                          plasma_enum_t uplo, plasma_desc_t A,
                                          int k, int mlo, int mhi)
{
    if (uplo != PlasmaLower || A.mb > NBMAX || A.mb != A.nb ||
        (A.precision != PlasmaRealDouble && A.precision != PlasmaRealFloat))
        return 0;
    int nk = plasma_tile_mview(A, k);
    int align = A.precision == PlasmaRealDouble ? 2 : 4;
    if (nk % PB != 0 || plasma_tile_mmain(A, k) % align != 0)
        return 0;
    if (mhi <= mlo)
        return 1;
    PLASMA_COUNT_LAUNCH();
    double rows = 0;
    for (int m = mlo; m < mhi; m++) rows += plasma_tile_mview(A, m);
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble)
        launch_trsm<double, 1>(s, st, A, k, mlo, mhi);
    else if (g_fp32_split == 1)
        launch_trsm<float, 1>(s, st, A, k, mlo, mhi);
    else
        launch_trsm<float, 3>(s, st, A, k, mlo, mhi);
    plasma_prof_end(prof, s, PLASMA_KCLASS_TRSM, rows * nk * nk,
                    2.0 * rows * nk * plasma_element_size(A.precision));
    return 1;
}
