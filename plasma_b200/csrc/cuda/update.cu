// update.cu -- trailing-matrix update of one Cholesky step:
//     A(m,n) -= A(m,k) * A(n,k)^T      for k < n <= m < mt,
// i.e. the SYRK on diagonal tiles and the GEMMs below them that the reference
// submits as nt(nt-1)/2 + C(nt,3) OpenMP tasks per factorisation
// (compute/pzpotrf.c:57-77 -> core_blas/core_zsyrk.c, core_zgemm.c:89-136).
//
// One persistent launch covers every tile of the step (or of a tile-column
// range, for look-ahead).  Work items are 128x128 sub-blocks of output
// tiles; each CTA walks the item list with a grid stride.  The strict upper
// part of diagonal tiles is never written (dsyrk with uplo = Lower leaves it
// untouched).
//
// FP64 lower storage: 8 warps of DMMA (mma.sync m16n8k8 f64, the FP64
// tensor-core path of sm_100 -- tcgen05 has no f64 kind), operands staged in
// shared memory by a 3-stage cp.async pipeline, accumulators in registers.
// FP32 (and the transposed upper-storage fallback): SIMT FFMA/DFMA 8x8
// register tiles.
#include "common.cuh"
#include "mma.cuh"

namespace {

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int THREADS = 256;

// Work item -> output tile (m,n) and sub-block (si,sj).
struct Item {
    int m, n, si, sj;
};

__device__ __forceinline__ bool decode_item(int w, int k, int nlo, int nhi,
                                            int mt, int sb, Item &it)
{
    int per = sb * sb;
    int p = w / per;
    int s = w - p * per;
    it.si = s / sb;
    it.sj = s - it.si * sb;
    int n = nlo;
    while (n < nhi && p >= mt - n) {
        p -= mt - n;
        n++;
    }
    if (n >= nhi) return false;
    it.n = n;
    it.m = n + p;
    (void)k;
    return true;
}

__host__ __device__ __forceinline__ long long count_items(int nlo, int nhi,
                                                          int mt, int sb)
{
    long long pairs = 0;
    for (int n = nlo; n < nhi; n++) pairs += mt - n;
    return pairs * sb * sb;
}

// ---------------------------------------------------------------------------
// FP64 DMMA kernel (lower storage, tiles column-major)
//
// CTA tile 128 x 64 (C rows x cols), 8 warps as 4 x 2, warp tile 32 x 32 =
// 2 x 4 m16n8k8 fragments; K streamed in chunks of 16 through a 4-stage
// cp.async ring.  At most 128 registers per thread so that two CTAs share an
// SM: one CTA's epilogue (a read-modify-write of C from HBM) overlaps the
// other's tensor-core main loop.  The C block is prefetched into L2 when the
// item starts, so the epilogue reads hit L2.
// ---------------------------------------------------------------------------
constexpr int DBM = 128;
constexpr int DBN = 64;
constexpr int DBK = 16;
constexpr int DSTAGES = 4;
constexpr int DPAD = 4;                 // row strides 132 / 68 doubles
constexpr int DLDS_A = DBM + DPAD;
constexpr int DLDS_B = DBN + DPAD;
constexpr int DSMEM = DSTAGES * DBK * (DLDS_A + DLDS_B) * (int)sizeof(double);

struct DmmaOperands {
    const double *a; int lda; int arows;   // A(m,k) logical rows
    const double *b; int ldb; int brows;   // A(n,k)
    int i0, j0, K;
    bool vec;                              // 16-byte copies are legal
};

__device__ __forceinline__ void dmma_load_stage(double *As, double *Bs,
                                                const DmmaOperands &op,
                                                int kc, int tid)
{
    if (op.vec) {
        // pairs of rows: A chunk 64 pairs x 16 cols, B chunk 32 pairs x 16
#pragma unroll
        for (int q = 0; q < (DBM * DBK / 2) / THREADS; q++) {
            int e = tid + q * THREADS;
            int r = 2 * (e % (DBM / 2)), c = e / (DBM / 2);
            int gi = op.i0 + r, gk = kc + c;
            bool v = gi < op.arows && gk < op.K;
            const double *src = v ? op.a + (size_t)gk * op.lda + gi : op.a;
            cp_async_16(As + c * DLDS_A + r, src, v);
        }
#pragma unroll
        for (int q = 0; q < (DBN * DBK / 2) / THREADS; q++) {
            int e = tid + q * THREADS;
            int r = 2 * (e % (DBN / 2)), c = e / (DBN / 2);
            int gj = op.j0 + r, gk = kc + c;
            bool v = gj < op.brows && gk < op.K;
            const double *src = v ? op.b + (size_t)gk * op.ldb + gj : op.b;
            cp_async_16(Bs + c * DLDS_B + r, src, v);
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < (DBM * DBK) / THREADS; q++) {
        int e = tid + q * THREADS;
        int r = e % DBM, c = e / DBM;
        int gi = op.i0 + r, gk = kc + c;
        bool v = gi < op.arows && gk < op.K;
        const double *src = v ? op.a + (size_t)gk * op.lda + gi : op.a;
        cp_async_8(As + c * DLDS_A + r, src, v);
    }
#pragma unroll
    for (int q = 0; q < (DBN * DBK) / THREADS; q++) {
        int e = tid + q * THREADS;
        int r = e % DBN, c = e / DBN;
        int gj = op.j0 + r, gk = kc + c;
        bool v = gj < op.brows && gk < op.K;
        const double *src = v ? op.b + (size_t)gk * op.ldb + gj : op.b;
        cp_async_8(Bs + c * DLDS_B + r, src, v);
    }
}

__global__ void __launch_bounds__(THREADS, 2)
k_update_dmma(plasma_desc_t A, int k, int nlo, int nhi, int nitems,
              const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (plasma_failed(st)) return;
    double *As = reinterpret_cast<double *>(smem_raw);
    double *Bs = As + DSTAGES * DBK * DLDS_A;

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp >> 1;          // 0..3 -> 32 rows each
    const int wn = warp & 1;           // 0..1 -> 32 cols each
    const int mt = A.mt;
    const int sbm = (A.mb + DBM - 1) / DBM;
    const int sbn = (A.mb + DBN - 1) / DBN;

    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        Item it;
        {
            int per = sbm * sbn;
            int p = w / per, s = w - p * per;
            it.si = s / sbn;
            it.sj = s - it.si * sbn;
            int n = nlo;
            while (n < nhi && p >= mt - n) { p -= mt - n; n++; }
            if (n >= nhi) break;
            it.n = n;
            it.m = n + p;
        }
        DmmaOperands op;
        op.i0 = it.si * DBM;
        op.j0 = it.sj * DBN;
        // a block of a diagonal tile that lies strictly above the diagonal
        if (it.m == it.n && op.j0 > op.i0 + DBM - 1) continue;
        op.a = (const double *)plasma_tile_addr(A, it.m, k);
        op.lda = plasma_tile_mmain(A, it.m);
        op.arows = plasma_tile_mview(A, it.m);
        op.b = (const double *)plasma_tile_addr(A, it.n, k);
        op.ldb = plasma_tile_mmain(A, it.n);
        op.brows = plasma_tile_mview(A, it.n);
        op.K = plasma_tile_nview(A, k);
        if (op.i0 >= op.arows || op.j0 >= op.brows) continue;
        op.vec = ((op.lda | op.ldb | op.arows | op.brows) & 1) == 0;

        double *C = (double *)plasma_tile_addr(A, it.m, it.n);
        const int ldc = plasma_tile_mmain(A, it.m);
        // warm L2 with the C block: 64 columns x 128 rows = 512 lines
        for (int e = tid; e < DBN * (DBM / 16); e += THREADS) {
            int j = op.j0 + e / (DBM / 16);
            int i = op.i0 + (e % (DBM / 16)) * 16;
            if (j < op.brows && i < op.arows)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(C + (size_t)j * ldc + i));
        }

        double acc[2][4][4];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 4; b++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][b][c] = 0.0;

        const int nk = (op.K + DBK - 1) / DBK;
        __syncthreads();   // previous item's readers are done with smem
#pragma unroll
        for (int s = 0; s < DSTAGES - 1; s++) {
            if (s < nk)
                dmma_load_stage(As + s * DBK * DLDS_A, Bs + s * DBK * DLDS_B,
                                op, s * DBK, tid);
            cp_async_commit();
        }
        for (int kt = 0; kt < nk; kt++) {
            cp_async_wait<DSTAGES - 2>();
            __syncthreads();
            int pf = kt + DSTAGES - 1;
            if (pf < nk) {
                int sl = pf % DSTAGES;
                dmma_load_stage(As + sl * DBK * DLDS_A, Bs + sl * DBK * DLDS_B,
                                op, pf * DBK, tid);
            }
            cp_async_commit();

            const double *as = As + (kt % DSTAGES) * DBK * DLDS_A + wm * 32;
            const double *bs = Bs + (kt % DSTAGES) * DBK * DLDS_B + wn * 32;
#pragma unroll
            for (int k8 = 0; k8 < DBK; k8 += 8) {
                double bf[4][2];
#pragma unroll
                for (int ni = 0; ni < 4; ni++) {
                    bf[ni][0] = bs[(k8 + t) * DLDS_B + ni * 8 + g];
                    bf[ni][1] = bs[(k8 + t + 4) * DLDS_B + ni * 8 + g];
                }
#pragma unroll
                for (int mi = 0; mi < 2; mi++) {
                    double af[4];
                    af[0] = as[(k8 + t) * DLDS_A + mi * 16 + g];
                    af[1] = as[(k8 + t) * DLDS_A + mi * 16 + g + 8];
                    af[2] = as[(k8 + t + 4) * DLDS_A + mi * 16 + g];
                    af[3] = as[(k8 + t + 4) * DLDS_A + mi * 16 + g + 8];
#pragma unroll
                    for (int ni = 0; ni < 4; ni++)
                        dmma_16x8x8(acc[mi][ni], af, bf[ni]);
                }
            }
        }
        cp_async_wait<0>();

        // epilogue: C -= acc.  All loads of one row fragment are issued
        // before any store so that their latencies overlap.
        const bool diag = it.m == it.n;
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            double cv[2][4][2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int i = op.i0 + wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        int j = op.j0 + wn * 32 + ni * 8 + 2 * t + e;
                        bool ok = i < op.arows && j < op.brows && (!diag || i >= j);
                        cv[h][ni][e] = ok ? C[(size_t)j * ldc + i] : 0.0;
                    }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int i = op.i0 + wm * 32 + mi * 16 + g + h * 8;
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        int j = op.j0 + wn * 32 + ni * 8 + 2 * t + e;
                        bool ok = i < op.arows && j < op.brows && (!diag || i >= j);
                        if (ok)
                            C[(size_t)j * ldc + i] = cv[h][ni][e] - acc[mi][ni][h * 2 + e];
                    }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Update step of a tile sweep with many right-hand sides (solve.cu):
//     B(m, :) -= a_m B(k, :)      for the row tiles m in [mlo, mhi)
// with a_m the factor block that couples tile row m with tile row k:
// L(m,k) (forward) or L(k,m)^T (backward), read from the storage triangle.
// Same core as k_update_dmma (128 x 64 CTA tiles, 8 warps, K in chunks of
// 16 through a 4-stage cp.async ring, two CTAs per SM): DMMA for FP64, the
// three-product TF32 split (FP32-accurate) for FP32.  The operands differ: the right-hand-side block b(kk, j) = B(k, :)(kk, j) is
// contiguous along K, and so is a_m when it is the transposed view.
// Those are copied element by element into the [K][row] stage layout (the
// shared-memory writes conflict, the tensor-core reads stay conflict-free).
// One work item = (row tile m, 128-row half, 64-column block of B).
// ---------------------------------------------------------------------------
struct SweepArgs {
    plasma_desc_t L, B;
    int uplo, trans;          // trans: backward sweep (L^T)
    int k, mlo, mhi;
    int sbm, ncb;             // row halves per tile, 64-column blocks of B
};

template <typename T>
struct SweepGeo {
    static constexpr int LDS_A = DBM + Pad<T>::v;   // conflict-free fragment reads
    static constexpr int LDS_B = DBN + Pad<T>::v;
    static constexpr int EPV = 16 / (int)sizeof(T); // elements per 16-byte copy
    static constexpr int SMEM = DSTAGES * DBK * (LDS_A + LDS_B) * (int)sizeof(T);
};

template <typename T>
__global__ void __launch_bounds__(THREADS, 2)
k_sweep_mma(SweepArgs g, int nitems, const plasma_devstat_t *st)
{
    using G = SweepGeo<T>;
    constexpr int LA = G::LDS_A, LB = G::LDS_B, EPV = G::EPV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (plasma_failed(st)) return;
    T *As = reinterpret_cast<T *>(smem_raw);
    T *Bs = As + DSTAGES * DBK * LA;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, t = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;
    const int nb = g.B.nb;
    const bool lower = g.uplo == PlasmaLower;
    // a_m contiguous along its rows (i) or along K
    const bool a_rows = lower ? !g.trans : g.trans;
    const int K = plasma_tile_mview(g.B, g.k);

    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const int jb = w % g.ncb;
        const int rest = w / g.ncb;
        const int si = rest % g.sbm;
        const int m = g.mlo + rest / g.sbm;
        const int i0 = si * DBM;
        const int rows = plasma_tile_mview(g.B, m);
        if (i0 >= rows) continue;
        const int jcol = jb * DBN;                    // first column of B
        const int jt = jcol / nb, jo = jcol - jt * nb;
        const int cols = min(DBN, plasma_tile_nview(g.B, jt) - jo);
        if (cols <= 0) continue;              // past a ragged last column tile

        // a_m(i, kk): the stored tile (m,k) with i contiguous (forward
        // lower: L(m,k); backward upper: U(m,k)), or the stored tile (k,m)
        // with kk contiguous (backward lower: L(k,m)^T; forward upper:
        // U(k,m)^T)
        const int am = a_rows ? m : g.k;
        const int an = a_rows ? g.k : m;
        const T *pa = (const T *)plasma_tile_addr(g.L, am, an);
        const int lda = plasma_tile_mmain(g.L, am);
        const T *pb = (const T *)plasma_tile_addr(g.B, g.k, jt) +
                           (size_t)jo * plasma_tile_mmain(g.B, g.k);
        const int ldb = plasma_tile_mmain(g.B, g.k);
        T *C = (T *)plasma_tile_addr(g.B, m, jt) +
                    (size_t)jo * plasma_tile_mmain(g.B, m);
        const int ldc = plasma_tile_mmain(g.B, m);
        const bool vec = a_rows && lda % EPV == 0 && rows % EPV == 0;

        auto load_stage = [&](int kc, int sl) {
            T *as = As + sl * DBK * LA;
            T *bs = Bs + sl * DBK * LB;
            if (vec) {
#pragma unroll
                for (int q = 0; q < (DBM * DBK / EPV) / THREADS; q++) {
                    const int e = tid + q * THREADS;
                    const int r = EPV * (e % (DBM / EPV)), c = e / (DBM / EPV);
                    const int gi = i0 + r, gk = kc + c;
                    const bool v = gi < rows && gk < K;
                    cp_async_16(as + c * LA + r, v ? pa + (size_t)gk * lda + gi : pa, v);
                }
            } else if (a_rows) {
#pragma unroll
                for (int q = 0; q < (DBM * DBK) / THREADS; q++) {
                    const int e = tid + q * THREADS;
                    const int r = e % DBM, c = e / DBM;
                    const int gi = i0 + r, gk = kc + c;
                    const bool v = gi < rows && gk < K;
                    cp_async_el(as + c * LA + r, v ? pa + (size_t)gk * lda + gi : pa, v);
                }
            } else {
                // a_m(i, kk) = tile[i * lda + kk]: lanes walk kk
#pragma unroll
                for (int q = 0; q < (DBM * DBK) / THREADS; q++) {
                    const int e = tid + q * THREADS;
                    const int c = e % DBK, r = e / DBK;
                    const int gi = i0 + r, gk = kc + c;
                    const bool v = gi < rows && gk < K;
                    cp_async_el(as + c * LA + r, v ? pa + (size_t)gi * lda + gk : pa, v);
                }
            }
            // b(kk, j) = B(k)(kk, jo + j) = pb[j * ldb + kk]: lanes walk kk
#pragma unroll
            for (int q = 0; q < (DBN * DBK) / THREADS; q++) {
                const int e = tid + q * THREADS;
                const int c = e % DBK, r = e / DBK;
                const int gk = kc + c;
                const bool v = r < cols && gk < K;
                cp_async_el(bs + c * LB + r, v ? pb + (size_t)r * ldb + gk : pb, v);
            }
        };

        T acc[2][4][4];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 4; b++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][b][c] = T(0);

        const int nk = (K + DBK - 1) / DBK;
        __syncthreads();   // the previous item's readers are done with smem
#pragma unroll
        for (int s = 0; s < DSTAGES - 1; s++) {
            if (s < nk) load_stage(s * DBK, s);
            cp_async_commit();
        }
        for (int kt = 0; kt < nk; kt++) {
            cp_async_wait<DSTAGES - 2>();
            __syncthreads();
            const int pf = kt + DSTAGES - 1;
            if (pf < nk) load_stage(pf * DBK, pf % DSTAGES);
            cp_async_commit();
            const T *as = As + (kt % DSTAGES) * DBK * LA + wm * 32;
            const T *bs = Bs + (kt % DSTAGES) * DBK * LB + wn * 32;
#pragma unroll
            for (int k8 = 0; k8 < DBK; k8 += 8) {
                T bf[4][2];
#pragma unroll
                for (int ni = 0; ni < 4; ni++) {
                    bf[ni][0] = bs[(k8 + t) * LB + ni * 8 + gq];
                    bf[ni][1] = bs[(k8 + t + 4) * LB + ni * 8 + gq];
                }
#pragma unroll
                for (int mi = 0; mi < 2; mi++) {
                    T af[4];
                    af[0] = as[(k8 + t) * LA + mi * 16 + gq];
                    af[1] = as[(k8 + t) * LA + mi * 16 + gq + 8];
                    af[2] = as[(k8 + t + 4) * LA + mi * 16 + gq];
                    af[3] = as[(k8 + t + 4) * LA + mi * 16 + gq + 8];
#pragma unroll
                    for (int ni = 0; ni < 4; ni++) mma8<3>(acc[mi][ni], af, bf[ni]);
                }
            }
        }
        cp_async_wait<0>();

        // C -= acc, all loads of a row fragment before its stores
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            T cv[2][4][2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = i0 + wm * 32 + mi * 16 + gq + h * 8;
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int j = wn * 32 + ni * 8 + 2 * t + e;
                        cv[h][ni][e] = (i < rows && j < cols) ? C[(size_t)j * ldc + i] : T(0);
                    }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = i0 + wm * 32 + mi * 16 + gq + h * 8;
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int j = wn * 32 + ni * 8 + 2 * t + e;
                        if (i < rows && j < cols)
                            C[(size_t)j * ldc + i] = cv[h][ni][e] - acc[mi][ni][h * 2 + e];
                    }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// SIMT kernel (FP32, or FP64 with transposed upper storage)
// ---------------------------------------------------------------------------
constexpr int SBK = 8;

template <typename T>
__global__ void __launch_bounds__(THREADS)
k_update_simt(plasma_desc_t A, int uplo, int k, int nlo, int nhi, int nitems,
              const plasma_devstat_t *st)
{
    __shared__ T As[SBK][BM + 4];
    __shared__ T Bs[SBK][BN + 4];
    if (plasma_failed(st)) return;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int mt = A.mt;
    const int sb = (A.mb + BM - 1) / BM;

    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        Item it;
        if (!decode_item(w, k, nlo, nhi, mt, sb, it)) break;
        if (it.m == it.n && it.sj > it.si) continue;
        TileView<T> a = tile_view<T>(A, uplo, it.m, k);
        TileView<T> b = tile_view<T>(A, uplo, it.n, k);
        TileView<T> c = tile_view<T>(A, uplo, it.m, it.n);
        const int i0 = it.si * BM, j0 = it.sj * BN;
        if (i0 >= a.rows || j0 >= b.rows) continue;
        const int K = a.cols;

        T acc[8][8];
#pragma unroll
        for (int x = 0; x < 8; x++)
#pragma unroll
            for (int y = 0; y < 8; y++) acc[x][y] = T(0);

        for (int kc = 0; kc < K; kc += SBK) {
            __syncthreads();
            for (int e = tid; e < BM * SBK; e += THREADS) {
                int r, cc;
                if (a.trans) { cc = e % SBK; r = e / SBK; }
                else         { r = e % BM;   cc = e / BM; }
                int gi = i0 + r, gk = kc + cc;
                As[cc][r] = (gi < a.rows && gk < K) ? a.at(gi, gk) : T(0);
                int gj = j0 + r;
                Bs[cc][r] = (gj < b.rows && gk < K) ? b.at(gj, gk) : T(0);
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < SBK; kk++) {
                T x[8], y[8];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    x[q] = As[kk][ty * 4 + q];
                    x[q + 4] = As[kk][64 + ty * 4 + q];
                    y[q] = Bs[kk][tx * 4 + q];
                    y[q + 4] = Bs[kk][64 + tx * 4 + q];
                }
#pragma unroll
                for (int p = 0; p < 8; p++)
#pragma unroll
                    for (int q = 0; q < 8; q++) acc[p][q] += x[p] * y[q];
            }
        }
        const bool diag = it.m == it.n;
#pragma unroll
        for (int p = 0; p < 8; p++) {
            int i = i0 + (p < 4 ? ty * 4 + p : 64 + ty * 4 + p - 4);
            if (i >= a.rows) continue;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                int j = j0 + (q < 4 ? tx * 4 + q : 64 + tx * 4 + q - 4);
                if (j < b.rows && (!diag || i >= j))
                    c.at(i, j) -= acc[p][q];
            }
        }
    }
}

}  // namespace

extern "C" void plasma_cuda_update(cudaStream_t s, plasma_devstat_t *st,
                                   plasma_enum_t uplo, plasma_desc_t A, int k,
                                   int nlo, int nhi, int num_sms)
{
    if (nhi <= nlo) return;
    const bool dmma = A.precision == PlasmaRealDouble && uplo == PlasmaLower;
    int sb = (A.mb + BM - 1) / BM;
    long long nitems = count_items(nlo, nhi, A.mt, sb);
    if (dmma) {
        long long pairs = count_items(nlo, nhi, A.mt, 1);
        nitems = pairs * ((A.mb + DBM - 1) / DBM) * ((A.mb + DBN - 1) / DBN);
    }
    if (nitems <= 0) return;
    PLASMA_COUNT_LAUNCH();
    // algorithmic work of this launch: SYRK on diagonal tiles, GEMM below
    double flops = 0.0, bytes = 0.0;
    {
        const double K = plasma_tile_nview(A, k);
        const double es = (double)plasma_element_size(A.precision);
        for (int n = nlo; n < nhi; n++) {
            double cn = plasma_tile_mview(A, n);
            for (int m = n; m < A.mt; m++) {
                double rm = plasma_tile_mview(A, m);
                flops += (m == n) ? cn * (cn + 1) * K : 2.0 * rm * cn * K;
                bytes += es * (m == n ? cn * (cn + 1) : 2.0 * rm * cn);
            }
        }
    }
    int prof = plasma_prof_begin(s);
    if (dmma) {
        static unsigned long long attr_set = 0;
        if (plasma_first_on_device(&attr_set)) {
            cudaFuncSetAttribute(k_update_dmma,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 DSMEM);
        }
        // one CTA per work item: SMs free up often, so the high-priority
        // critical-path kernels of the next step are scheduled in between
        long long grid = nitems;
        (void)num_sms;
        k_update_dmma<<<(unsigned)grid, THREADS, DSMEM, s>>>(
            A, k, nlo, nhi, (int)nitems, st);
    } else {
        long long grid = nitems;     // one CTA per item (see above)
        if (A.precision == PlasmaRealDouble)
            k_update_simt<double><<<(unsigned)grid, THREADS, 0, s>>>(
                A, uplo, k, nlo, nhi, (int)nitems, st);
        else
            k_update_simt<float><<<(unsigned)grid, THREADS, 0, s>>>(
                A, uplo, k, nlo, nhi, (int)nitems, st);
    }
    plasma_prof_end(prof, s, PLASMA_KCLASS_UPDATE, flops, bytes);
}

// One update step of a tile sweep with many right-hand sides (see
// k_sweep_mma): B rows of tiles [mlo, mhi) -= the factor block coupling them
// with tile row k times B(k, :).  FP64 on DMMA, FP32 as three TF32
// products.  Returns 0 (nothing launched) when the tiling does not fit
// (square tiles, a multiple of 128).
extern "C" int plasma_cuda_sweep_update_mma(cudaStream_t s, plasma_devstat_t *st,
                                            plasma_enum_t uplo, int trans,
                                            plasma_desc_t L, plasma_desc_t B, int k,
                                            int mlo, int mhi)
{
    if (L.precision != B.precision ||
        (L.precision != PlasmaRealDouble && L.precision != PlasmaRealFloat) ||
        L.mb != L.nb || B.mb != L.mb || B.nb != L.nb || L.mb % DBM != 0 ||
        L.i != 0 || L.j != 0 || B.i != 0 || B.j != 0)
        return 0;
    if (mhi <= mlo || B.n == 0) return 1;
    SweepArgs g;
    g.L = L;
    g.B = B;
    g.uplo = uplo;
    g.trans = trans;
    g.k = k;
    g.mlo = mlo;
    g.mhi = mhi;
    g.sbm = L.mb / DBM;
    // 64-column blocks per column tile, times the column tiles
    g.ncb = ((B.nb + DBN - 1) / DBN) * B.nt;
    const long long nitems = (long long)(mhi - mlo) * g.sbm * g.ncb;
    PLASMA_COUNT_LAUNCH();
    if (L.precision == PlasmaRealDouble) {
        static unsigned long long attr = 0;
        if (plasma_first_on_device(&attr)) {
            cudaFuncSetAttribute(k_sweep_mma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SweepGeo<double>::SMEM);
        }
        k_sweep_mma<double><<<(unsigned)nitems, THREADS, SweepGeo<double>::SMEM, s>>>(
            g, (int)nitems, st);
    } else {
        static unsigned long long attr = 0;
        if (plasma_first_on_device(&attr)) {
            cudaFuncSetAttribute(k_sweep_mma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SweepGeo<float>::SMEM);
        }
        k_sweep_mma<float><<<(unsigned)nitems, THREADS, SweepGeo<float>::SMEM, s>>>(
            g, (int)nitems, st);
    }
    return 1;
}
