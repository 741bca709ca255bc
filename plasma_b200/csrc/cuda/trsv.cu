// trsv.cu -- one-launch triangular sweeps with a tile Cholesky factor for a
// single right-hand side (the two plasma_pdtrsm sweeps of potrs,
// compute/pztrsm.c:113-177, as used by every refinement step of dsposv).
//
// The sweep walks blocks of SB rows (SB = 128 for FP32 factors, 64 for FP64;
// a storage tile holds nb/SB of them):
//   forward  (L y = b):   y_u = W_u (b_u - sum_{k<u} L(u,k) y_k)
//   backward (L^T x = y): x_u = W_u^T (y_u - sum_{k>u} L(k,u)^T x_k)
// with W_u the inverse of the SB x SB diagonal block (k_trtri_blocks).
//
// One persistent kernel per sweep.  CTAs take blocks in sweep order from an
// atomic ticket; block u consumes the blocks of earlier tickets as their
// ready flags appear (each flag is the sweep's epoch, written after the block
// and a fence).  A CTA only ever waits for blocks taken before its own, by
// CTAs that are already running, so the sweep cannot deadlock.  The chain of
// the sweep runs through the coupling of u with the block just before it;
// that block of L and W_u are copied into shared memory as soon as the CTA
// takes u, so the step on the chain reads shared memory only.  Every wait is
// bounded (about 2 s): on expiry the CTA sets a shared abort word and the
// device status (PlasmaErrorInternal), and all CTAs leave.
//
// Lower storage: L(i,j) is element (i,j) of tile (i/nb, j/nb).  Upper storage
// (A = U^T U): L(i,j) = U(j,i).
#include "common.cuh"

namespace {

constexpr int TS_THREADS = 256;

struct SweepSync {
    int ticket;
    int abort;
    int flags[1];          // [nblk]
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ bool wait_block(SweepSync *sy, int k, int epoch)
{
    long long t0 = clock64();
    while (ld_acquire(&sy->flags[k]) != epoch) {
        if (ld_acquire(&sy->abort)) return false;
        if (clock64() - t0 > 4000000000LL) {
            atomicExch(&sy->abort, 1);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

template <typename T>
__device__ __forceinline__ void cp_async_el_any(T *dst, const T *src)
{
    if (sizeof(T) == 8) cp_async_8(dst, src, true);
    else cp_async_4(dst, src, true);
}

// as above; valid = false writes zero and reads nothing (src must still be
// a global address)
template <typename T>
__device__ __forceinline__ void cp_async_el_any_z(T *dst, const T *src, bool valid)
{
    if (sizeof(T) == 8) cp_async_8(dst, src, valid);
    else cp_async_4(dst, src, valid);
}

// Logical block (bi, bj) of L, SB x SB: element (i,j) at p[i*si + j*sj].
template <typename T>
struct LBlock {
    const T *p;
    int si, sj;
};

template <typename T, int SB>
__device__ __forceinline__ LBlock<T> lblock(const plasma_desc_t &A, bool lower,
                                            int bi, int bj)
{
    const int gi = bi * SB, gj = bj * SB;
    const int ti = gi / A.mb, tj = gj / A.mb;
    const int oi = gi % A.mb, oj = gj % A.mb;
    LBlock<T> b;
    if (lower) {
        const T *t = (const T *)plasma_tile_addr(A, ti, tj);
        int ld = plasma_tile_mmain(A, ti);
        b.p = t + (size_t)oj * ld + oi;
        b.si = 1;
        b.sj = ld;
    } else {
        const T *t = (const T *)plasma_tile_addr(A, tj, ti);
        int ld = plasma_tile_mmain(A, tj);
        b.p = t + (size_t)oi * ld + oj;
        b.si = ld;
        b.sj = 1;
    }
    return b;
}

// ys[i] -= sum_c M(i,c) xs[c] for i < rows, c < cols, M(i,c) = m[i*si + c*sj].
// TS_THREADS / SB threads per row, each a share of the columns, 32 loads in
// flight per thread; shares meet in shared memory.
template <typename T, int SB>
__device__ __forceinline__ void gemv_n(const T *m, int si, int sj, int rows, int cols,
                                       const T *xs, T *ys, T *red, int tid)
{
    static_assert(2 * SB <= TS_THREADS, "at least two threads per row");
    constexpr int NH = TS_THREADS / SB;
    const int i = tid % SB, h = tid / SB;
    T s = 0;
    if (i < rows) {
        const int share = (cols + NH - 1) / NH;
        const int c0 = h * share;
        const int c1 = min(cols, c0 + share);
        int c = c0;
        for (; c + 32 <= c1; c += 32) {
            T a[32];
#pragma unroll
            for (int q = 0; q < 32; q++) a[q] = m[(size_t)i * si + (size_t)(c + q) * sj];
#pragma unroll
            for (int q = 0; q < 32; q++) s += a[q] * xs[c + q];
        }
        for (; c < c1; c++) s += m[(size_t)i * si + (size_t)c * sj] * xs[c];
    }
    red[h * SB + i] = s;
    __syncthreads();
    if (tid < rows) {
        T t = 0;
#pragma unroll
        for (int q = 0; q < NH; q++) t += red[q * SB + tid];
        ys[tid] -= t;
    }
    __syncthreads();
}

// ys[j] -= sum_r M(r,j) xs[r] for j < cols, r < rows, M(r,j) = m[r + j*sj]
// (rows contiguous): warps own 32-column groups and a share of the rows;
// lanes walk rows (coalesced), a butterfly reduces the column sums across
// lanes, and the row shares meet in shared memory.
template <typename T, int SB>
__device__ __forceinline__ void gemv_t(const T *m, int sj, int rows, int cols,
                                       const T *xs, T *ys, T *red, int lane, int warp,
                                       int tid)
{
    constexpr int NW = TS_THREADS / 32;
    constexpr int CG = SB / 32;                    // column groups
    constexpr int RS = NW / CG;                    // row shares
    const int cg = warp % CG, rs = warp / CG;
    T v[32];
#pragma unroll
    for (int c = 0; c < 32; c++) v[c] = 0;
    const int rchunk = (rows + RS - 1) / RS;
    const int r0 = rs * rchunk, r1 = min(rows, r0 + rchunk);
    for (int r = r0 + lane; r < r1; r += 32) {
        const T xr = xs[r];
#pragma unroll
        for (int c = 0; c < 32; c++) {
            int col = cg * 32 + c;
            v[c] += (col < cols ? m[(size_t)r + (size_t)col * sj] : T(0)) * xr;
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool hi = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < off; i++) {
            T send = hi ? v[i] : v[i + off];
            T keep = hi ? v[i + off] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    red[rs * SB + cg * 32 + lane] = v[0];
    __syncthreads();
    if (tid < cols) {
        T t = 0;
#pragma unroll
        for (int q = 0; q < RS; q++) t += red[q * SB + tid];
        ys[tid] -= t;
    }
    __syncthreads();
}

template <typename T, int SB>
__global__ void __launch_bounds__(TS_THREADS, 1)
k_trsv(plasma_desc_t A, int uplo, int backward, const T *W, T *vec,
       SweepSync *sy, int epoch, plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Lc = reinterpret_cast<T *>(smem_raw);        // critical block, [c*SB + i]
    T *Wc = Lc + SB * SB;                           // W_u, [c*SB + i]
    T *xs = Wc + SB * SB;
    T *ys = xs + SB;
    T *tmp = ys + SB;
    T *red = tmp + SB;                              // TS_THREADS entries
    __shared__ int blk_s, ok_s;
    if (plasma_failed(st)) return;
    const int n = A.m;
    const int nblk = (n + SB - 1) / SB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool lower = uplo == PlasmaLower;

    for (;;) {
        if (tid == 0) blk_s = atomicAdd(&sy->ticket, 1);
        __syncthreads();
        const int t = blk_s;
        __syncthreads();
        if (t >= nblk) break;
        const int u = backward ? nblk - 1 - t : t;
        const int rows = min(SB, n - u * SB);

        // stage W_u and the critical block (the coupling with the block of
        // ticket t-1) in shared memory; both are read-only factor data
        const T *wu = W + (size_t)u * SB * SB;
        for (int e = tid; e < SB * SB; e += TS_THREADS)
            cp_async_el_any(Wc + e, wu + e);
        const int kc = t > 0 ? (backward ? u + 1 : u - 1) : -1;
        const int kcr = kc >= 0 ? min(SB, n - kc * SB) : 0;
        if (kc >= 0) {
            // logical block stored as Lc[c*SB + i]:
            //   forward : L(u, kc), i < rows, c < kcr
            //   backward: L(kc, u), i < kcr,  c < rows
            LBlock<T> b = backward ? lblock<T, SB>(A, lower, kc, u)
                                   : lblock<T, SB>(A, lower, u, kc);
            const int ri = backward ? kcr : rows, rc = backward ? rows : kcr;
            for (int e = tid; e < SB * SB; e += TS_THREADS) {
                int i = e % SB, c = e / SB;
                if (i < ri && c < rc)
                    cp_async_el_any(Lc + e, b.p + (size_t)i * b.si + (size_t)c * b.sj);
                else
                    Lc[e] = T(0);
            }
        }
        cp_async_commit();
        for (int i = tid; i < SB; i += TS_THREADS)
            ys[i] = i < rows ? vec[(size_t)u * SB + i] : T(0);

        for (int s = 0; s < t; s++) {
            const int k = backward ? nblk - 1 - s : s;
            const int kr = min(SB, n - k * SB);
            if (tid == 0) {
                ok_s = wait_block(sy, k, epoch) ? 1 : 0;
                if (!ok_s) plasma_fail(st, PlasmaErrorInternal, 0);
            }
            __syncthreads();
            if (!ok_s) {
                cp_async_wait<0>();
                return;
            }
            for (int i = tid; i < SB; i += TS_THREADS)
                xs[i] = i < kr ? ((volatile T *)vec)[(size_t)k * SB + i] : T(0);
            if (s == t - 1) cp_async_wait<0>();
            __syncthreads();
            if (s == t - 1) {
                if (!backward) gemv_n<T, SB>(Lc, 1, SB, rows, kr, xs, ys, red, tid);
                else gemv_t<T, SB>(Lc, SB, kr, rows, xs, ys, red, lane, warp, tid);
            } else {
                LBlock<T> b = backward ? lblock<T, SB>(A, lower, k, u)
                                       : lblock<T, SB>(A, lower, u, k);
                if (!backward) {
                    gemv_n<T, SB>(b.p, b.si, b.sj, rows, kr, xs, ys, red, tid);
                } else if (b.si == 1) {
                    gemv_t<T, SB>(b.p, b.sj, kr, rows, xs, ys, red, lane, warp, tid);
                } else {
                    // upper storage, backward: L(k,u)^T = U(u,k), a plain
                    // column-major block -> forward form
                    gemv_n<T, SB>(b.p, b.sj, b.si, rows, kr, xs, ys, red, tid);
                }
            }
        }
        if (t == 0) cp_async_wait<0>();
        __syncthreads();
        // diagonal block: ys <- W_u ys (forward) or W_u^T ys (backward)
        for (int i = tid; i < SB; i += TS_THREADS) {
            tmp[i] = -ys[i];
            ys[i] = 0;
        }
        __syncthreads();
        if (!backward) gemv_n<T, SB>(Wc, 1, SB, rows, rows, tmp, ys, red, tid);
        else gemv_t<T, SB>(Wc, SB, rows, rows, tmp, ys, red, lane, warp, tid);
        for (int i = tid; i < rows; i += TS_THREADS) vec[(size_t)u * SB + i] = ys[i];
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(&sy->flags[u], epoch);
    }
}

// W_u = inv(logical L diagonal block u, SB x SB), written densely
// ([u][c*SB + i]); rows and columns beyond the matrix are the identity.
// unit: the diagonal of L is taken as one (the unit-lower factor of an LU).
template <typename T, int SB>
__global__ void __launch_bounds__(256)
k_trtri_blocks(plasma_desc_t A, int uplo, int unit, T *W, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ls = reinterpret_cast<T *>(smem_raw);       // [SB][SB+1]
    T *S = Ls + SB * (SB + 1);                     // [SB][33]
    if (plasma_failed(st)) return;
    const int u = blockIdx.x, n = A.m;
    const int rows = min(SB, n - u * SB);
    LBlock<T> b = lblock<T, SB>(A, uplo == PlasmaLower, u, u);
    const int tid = threadIdx.x;
    for (int e = tid; e < SB * SB; e += 256) {
        int i = e % SB, c = e / SB;
        Ls[c * (SB + 1) + i] = (i < rows && c < rows && i >= c && !(unit && i == c))
            ? b.p[(size_t)i * b.si + (size_t)c * b.sj] : (i == c ? T(1) : T(0));
    }
    __syncthreads();
    T *w = W + (size_t)u * SB * SB;
    // solve L Wcol = e for 32 columns at a time, right-looking
    for (int c0 = 0; c0 < SB; c0 += 32) {
        for (int e = tid; e < SB * 32; e += 256) {
            int i = e % SB, c = e / SB;
            S[i * 33 + c] = (i == c0 + c) ? T(1) : T(0);
        }
        __syncthreads();
        for (int j = c0; j < SB; j++) {
            T rjj = T(1) / Ls[j * (SB + 1) + j];
            if (tid < 32) S[j * 33 + tid] *= rjj;
            __syncthreads();
            for (int e = tid; e < (SB - j - 1) * 32; e += 256) {
                int i = j + 1 + e / 32, c = e % 32;
                S[i * 33 + c] -= Ls[j * (SB + 1) + i] * S[j * 33 + c];
            }
            __syncthreads();
        }
        for (int e = tid; e < SB * 32; e += 256) {
            int i = e % SB, c = e / SB;
            w[(size_t)(c0 + c) * SB + i] = S[i * 33 + c];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// One-launch sweeps for a few right-hand sides (potrs / posv with
// 2 <= nrhs <= 32; the reference runs them as the tile tasks of pztrsm.c):
// the ticketed row blocks of k_trsv, each applied to NR columns of B at
// once, so the factor is read once per NR columns instead of once per
// column, and B stays in its tile layout.
//   forward : X_u = W_u   (B_u - sum_{k<u} L(u,k) X_k)
//   backward: X_u = W_u^T (B_u - sum_{k>u} L(k,u)^T X_k)
// Block u streams the operator blocks of the earlier tickets through a
// two-deep cp.async ring in shared memory, stored as Ms[c*(SB+1) + i] =
// M(i,c) whatever the storage order of L (the global reads are coalesced
// along whichever index is contiguous).  Thread (i, h) owns row i and the
// h-th share of the columns c of the operator and keeps its NR partial sums
// in registers across all blocks k; the shares meet in shared memory once,
// before the diagonal block.  Solution blocks of other CTAs are read
// through L2 (ld.global.cg) after their ready flag.
// ---------------------------------------------------------------------------
constexpr int TR_THREADS = 256;

template <typename T, int SB, int NR>
constexpr int trsm_rows_smem()
{
    return (2 * SB * (SB + 1) + SB * NR + (TR_THREADS / SB) * SB * NR) * (int)sizeof(T);
}

template <typename T>
__device__ __forceinline__ T *b_elem(const plasma_desc_t &B, int row, int col)
{
    const int m = row / B.mb, r = row - m * B.mb;
    const int t = col / B.nb, c = col - t * B.nb;
    return (T *)plasma_tile_addr(B, m, t) + (size_t)c * plasma_tile_mmain(B, m) + r;
}

// Ms[c*(SB+1) + i] <- q[i*mi + c*mc] for i < ri, c < rc, zero elsewhere
template <typename T, int SB>
__device__ __forceinline__ void stage_op(T *Ms, const T *q, int mi, int mc, int ri, int rc,
                                         int tid)
{
    constexpr int LDM = SB + 1;
    if (mi == 1) {
        for (int e = tid; e < SB * SB; e += TR_THREADS) {
            const int i = e % SB, c = e / SB;
            const bool v = i < ri && c < rc;
            cp_async_el_any_z(Ms + c * LDM + i, v ? q + (size_t)i + (size_t)c * mc : q, v);
        }
    } else {
        for (int e = tid; e < SB * SB; e += TR_THREADS) {
            const int c = e % SB, i = e / SB;
            const bool v = i < ri && c < rc;
            cp_async_el_any_z(Ms + c * LDM + i, v ? q + (size_t)i * mi + (size_t)c : q, v);
        }
    }
}

template <typename T, int SB, int NR>
__global__ void __launch_bounds__(TR_THREADS, 1)
k_trsm_rows(plasma_desc_t A, int uplo, int backward, const T *W, plasma_desc_t B,
            int c0, int ncols, SweepSync *sy, int epoch, plasma_devstat_t *st)
{
    constexpr int LDM = SB + 1;
    constexpr int SH = TR_THREADS / SB;      // column shares
    constexpr int CS = SB / SH;              // columns of the operator per share
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ms[2] = {reinterpret_cast<T *>(smem_raw),
                reinterpret_cast<T *>(smem_raw) + SB * LDM};
    T *Xs = Ms[1] + SB * LDM;                // [SB][NR]
    T *red = Xs + SB * NR;                   // [SH][SB][NR]
    __shared__ int blk_s, ok_s;
    if (plasma_failed(st)) return;
    const int n = A.m;
    const int nblk = (n + SB - 1) / SB;
    const int tid = threadIdx.x;
    const int i = tid % SB, h = tid / SB;
    const bool lower = uplo == PlasmaLower;

    for (;;) {
        if (tid == 0) blk_s = atomicAdd(&sy->ticket, 1);
        __syncthreads();
        const int t = blk_s;
        __syncthreads();
        if (t >= nblk) break;
        const int u = backward ? nblk - 1 - t : t;
        const int rows = min(SB, n - u * SB);

        // operator of ticket s: forward L(u,k), backward L(k,u)^T
        auto stage = [&](int s, T *buf) {
            const int k = backward ? nblk - 1 - s : s;
            const int kr = min(SB, n - k * SB);
            if (!backward) {
                LBlock<T> b = lblock<T, SB>(A, lower, u, k);
                stage_op<T, SB>(buf, b.p, b.si, b.sj, rows, kr, tid);
            } else {
                LBlock<T> b = lblock<T, SB>(A, lower, k, u);
                stage_op<T, SB>(buf, b.p, b.sj, b.si, rows, kr, tid);
            }
        };
        T acc[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) acc[j] = T(0);
        if (t > 0) stage(0, Ms[0]);
        cp_async_commit();
        for (int s = 0; s < t; s++) {
            const int k = backward ? nblk - 1 - s : s;
            const int kr = min(SB, n - k * SB);
            if (s + 1 < t) stage(s + 1, Ms[(s + 1) & 1]);
            cp_async_commit();
            if (tid == 0) {
                ok_s = wait_block(sy, k, epoch) ? 1 : 0;
                if (!ok_s) plasma_fail(st, PlasmaErrorInternal, 0);
            }
            __syncthreads();
            if (!ok_s) {
                cp_async_wait<0>();
                return;
            }
            for (int e = tid; e < SB * NR; e += TR_THREADS) {
                const int r = e / NR, j = e - (e / NR) * NR;
                Xs[e] = (r < kr && j < ncols) ? __ldcg(b_elem<T>(B, k * SB + r, c0 + j)) : T(0);
            }
            cp_async_wait<1>();
            __syncthreads();
            const T *Mb = Ms[s & 1];
#pragma unroll 4
            for (int c = h * CS; c < (h + 1) * CS; c++) {
                const T m = Mb[c * LDM + i];
#pragma unroll
                for (int j = 0; j < NR; j++) acc[j] += m * Xs[c * NR + j];
            }
            __syncthreads();
        }
        cp_async_wait<0>();
        // the diagonal block's operator: W_u (forward) or W_u^T (backward)
        const T *wu = W + (size_t)u * SB * SB;
        if (!backward) stage_op<T, SB>(Ms[0], wu, 1, SB, SB, SB, tid);
        else stage_op<T, SB>(Ms[0], wu, SB, 1, SB, SB, tid);
        cp_async_commit();
#pragma unroll
        for (int j = 0; j < NR; j++) red[(h * SB + i) * NR + j] = acc[j];
        __syncthreads();
        for (int e = tid; e < SB * NR; e += TR_THREADS) {
            const int r = e / NR, j = e - (e / NR) * NR;
            T v = (r < rows && j < ncols) ? *b_elem<T>(B, u * SB + r, c0 + j) : T(0);
#pragma unroll
            for (int q = 0; q < SH; q++) v -= red[(q * SB + r) * NR + j];
            Xs[e] = v;
        }
        cp_async_wait<0>();
        __syncthreads();
#pragma unroll
        for (int j = 0; j < NR; j++) acc[j] = T(0);
#pragma unroll 4
        for (int c = h * CS; c < (h + 1) * CS; c++) {
            const T m = Ms[0][c * LDM + i];
#pragma unroll
            for (int j = 0; j < NR; j++) acc[j] += m * Xs[c * NR + j];
        }
#pragma unroll
        for (int j = 0; j < NR; j++) red[(h * SB + i) * NR + j] = acc[j];
        __syncthreads();
        for (int e = tid; e < SB * NR; e += TR_THREADS) {
            const int r = e / NR, j = e - (e / NR) * NR;
            if (r < rows && j < ncols) {
                T v = T(0);
#pragma unroll
                for (int q = 0; q < SH; q++) v += red[(q * SB + r) * NR + j];
                *b_elem<T>(B, u * SB + r, c0 + j) = v;
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(&sy->flags[u], epoch);
    }
}

template <typename T, int SB, int NR>
void launch_trsm_rows(cudaStream_t s, plasma_devstat_t *st, int uplo, int backward,
                      const plasma_desc_t &A, const void *W, const plasma_desc_t &B, int c0,
                      int ncols, SweepSync *sy, int epoch, int grid)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsm_rows<T, SB, NR>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trsm_rows_smem<T, SB, NR>());
    }
    k_trsm_rows<T, SB, NR><<<grid, TR_THREADS, trsm_rows_smem<T, SB, NR>(), s>>>(
        A, uplo, backward, (const T *)W, B, c0, ncols, sy, epoch, st);
}

// ---------------------------------------------------------------------------
// FP32 sweeps with 128-row blocks (the refinement sweeps of dsposv): the
// same ticketed row blocks, restructured so that neither the streaming of
// the factor nor the chain of blocks waits on the other.
//
//  * Off the chain: block u accumulates s_u = sum_k L(u,k) y_k over the
//    blocks k before u-1 (after u+1 backward).  Each of 512 threads owns 32
//    elements of every such block, and three blocks are in flight in
//    registers: block j+3 is requested as soon as block j is consumed, so
//    the factor streams while the CTA waits for solution blocks, and the
//    partial sums stay in registers until the row is done (one reduction
//    per row).  Then q_u = W_u (b_u - s_u) from shared memory.
//  * On the chain: y_u = q_u - M_u y_{u-1}, M_u = W_u L(u,u-1) precomputed
//    per factor (backward: M_u = W_u^T L(u+1,u)^T), one 128 x 128
//    matrix-vector product from shared memory.
//  * Publication: y_u goes out as 64-bit words (value, epoch), each one
//    single-copy atomic, which the consumers poll element by element: no
//    fence and no separate ready flag between the last store of a block and
//    its first use.  The epoch is the sweep's; the words of earlier sweeps
//    carry older epochs.
// The factor blocks are read in one of two shapes: "N", element (i,c) at
// p[i + c*ld] (rows of the result contiguous: forward lower, backward
// upper), or "T", element (r,i) at p[r + i*ld] (forward upper, backward
// lower).  Every wait is bounded as in k_trsv.
// ---------------------------------------------------------------------------
constexpr int LL_SB = 128;

struct Couple {
    // per block u, SB x SB column-major ([c*SB + i]): Wf = inv(L_uu),
    // Wb = Wf^T, Mf = Wf L(u,u-1), Mb = Wf^T L(u+1,u)^T
    const float *Wf, *Wb, *Mf, *Mb;
};

__device__ __forceinline__ unsigned long long ll_pack(float v, int epoch)
{
    return ((unsigned long long)(unsigned)epoch << 32) | (unsigned long long)__float_as_uint(v);
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Thread tid < SB waits for element tid of block k (rows beyond kr read as
// 0) and leaves it in ys; false when the sweep gave up.
__device__ __forceinline__ unsigned long long ll_peek(const unsigned long long *ll, int k,
                                                      int kr, int tid)
{
    return (tid < kr) ? ld_relaxed_u64(ll + (size_t)k * LL_SB + tid) : 0ull;
}

// w: the word already read for this element (ll_peek), re-read until its
// epoch is the sweep's
__device__ __forceinline__ bool ll_fetch(const unsigned long long *ll, SweepSync *sy, int k,
                                         int kr, int epoch, float *ys, int tid,
                                         int *abort_s, unsigned long long w)
{
    if (tid < LL_SB) {
        float v = 0.f;
        if (tid < kr) {
            const unsigned long long *p = ll + (size_t)k * LL_SB + tid;
            if ((int)(w >> 32) != epoch) {
                // one load per poll on the chain; the abort word and the
                // clock are looked at every 64 polls
                const long long t0 = clock64();
                for (int it = 1;; it++) {
                    w = ld_relaxed_u64(p);
                    if ((int)(w >> 32) == epoch) break;
                    if ((it & 63) == 0) {
                        if (*(volatile int *)abort_s ||
                            *(volatile const int *)&sy->abort) {
                            *(volatile int *)abort_s = 1;
                            break;
                        }
                        if (clock64() - t0 > 4000000000LL) {
                            atomicExch(&sy->abort, 1);
                            *(volatile int *)abort_s = 1;
                            break;
                        }
                    }
                }
            }
            v = __uint_as_float((unsigned)w);
        }
        ys[tid] = v;
    }
    __syncthreads();
    return *(volatile int *)abort_s == 0;
}

// 512 threads; each owns 32 elements of every coupling block.
constexpr int LL_THREADS = 512;
constexpr int LL_PER = LL_SB * LL_SB / LL_THREADS;   // 32
static_assert(LL_PER == 32 && LL_THREADS / 32 * 8 == LL_SB, "block shape");

// Both shapes move the block with 16-byte loads: a thread owns four
// consecutive rows (the contiguous index) of eight columns, a warp reads
// 512 contiguous bytes per load.  Full, aligned blocks take the
// unpredicated path.
//
// Shape N: element (i,c) at p[i + c*ld]; thread t owns rows 4(t%32) .. +3
// of columns 8(t/32) .. +7: a[j] = rows of column 8(t/32) + j.
__device__ __forceinline__ void load_n(const float *p, int ld, int rows, int cols, int tid,
                                       float4 (&a)[8])
{
    const int i0 = 4 * (tid & 31), c0 = 8 * (tid >> 5);
    // 16-byte loads need a full block, a 16-byte aligned start and a
    // leading dimension that keeps every column aligned (ragged last
    // tiles may have any leading dimension)
    if (rows == LL_SB && cols == LL_SB && (ld & 3) == 0 && ((uintptr_t)p & 15) == 0) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            a[j] = __ldg(reinterpret_cast<const float4 *>(p + i0 + (size_t)(c0 + j) * ld));
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float *q = p + i0 + (size_t)(c0 + j) * ld;
            const bool cj = c0 + j < cols;
            a[j].x = (cj && i0 < rows) ? __ldg(q) : 0.f;
            a[j].y = (cj && i0 + 1 < rows) ? __ldg(q + 1) : 0.f;
            a[j].z = (cj && i0 + 2 < rows) ? __ldg(q + 2) : 0.f;
            a[j].w = (cj && i0 + 3 < rows) ? __ldg(q + 3) : 0.f;
        }
    }
}

// acc[q] (row 4(t%32) + q) += sum_j a[j].q * y[8(t/32) + j]
__device__ __forceinline__ void fma_n(const float4 (&a)[8], const float *ys, int tid,
                                      float (&acc)[8])
{
    const int c0 = 8 * (tid >> 5);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float y = ys[c0 + j];
        acc[0] += a[j].x * y;
        acc[1] += a[j].y * y;
        acc[2] += a[j].z * y;
        acc[3] += a[j].w * y;
    }
}

// Shape T: element (r,i) at p[r + i*ld]; thread t owns rows 4(t%32) .. +3
// (the summed index) of result columns 8(t/32) .. +7.
__device__ __forceinline__ void load_t(const float *p, int ld, int rrows, int icols, int tid,
                                       float4 (&a)[8])
{
    load_n(p, ld, rrows, icols, tid, a);
}

// acc[j] (result column 8(t/32) + j) += sum_q a[j].q * y[4(t%32) + q]
__device__ __forceinline__ void fma_t(const float4 (&a)[8], const float *ys, int tid,
                                      float (&acc)[8])
{
    const float4 y = *reinterpret_cast<const float4 *>(ys + 4 * (tid & 31));
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] += a[j].x * y.x + a[j].y * y.y + a[j].z * y.z + a[j].w * y.w;
}

// out[i] = sum_c M[c*SB + i] v[c] for i < SB: shape N from shared memory,
// the four column quarters meeting in red (512 floats); result valid for
// tid < SB after the call.
__device__ __forceinline__ float smem_gemv(const float *M, const float *v, float *red, int tid)
{
    const int i = tid & 127, c0 = (tid >> 7) * LL_PER;
    float s = 0.f;
#pragma unroll 16
    for (int q = 0; q < LL_PER; q++) s += M[(c0 + q) * LL_SB + i] * v[c0 + q];
    red[tid] = s;
    __syncthreads();
    float r = 0.f;
    if (tid < LL_SB) r = red[tid] + red[LL_SB + tid] + red[2 * LL_SB + tid] + red[3 * LL_SB + tid];
    __syncthreads();
    return r;
}

template <bool SHAPE_T>
__device__ __forceinline__ void row_block_addr(const plasma_desc_t &A, bool lower,
                                               bool backward, int u, int k,
                                               const float *&p, int &ld)
{
    // the block of the factor that couples row block u with block k:
    // forward L(u,k), backward L(k,u); stored in the tile of the storage
    // triangle that holds it
    const int bi = backward ? k : u, bj = backward ? u : k;   // logical L(bi,bj)
    const int gi = bi * LL_SB, gj = bj * LL_SB;
    const int ti = gi / A.mb, tj = gj / A.mb, oi = gi % A.mb, oj = gj % A.mb;
    if (lower) {
        const float *t = (const float *)plasma_tile_addr(A, ti, tj);
        ld = plasma_tile_mmain(A, ti);
        p = t + (size_t)oj * ld + oi;        // L(bi,bj)(r,c) at p[r + c*ld]
    } else {
        const float *t = (const float *)plasma_tile_addr(A, tj, ti);
        ld = plasma_tile_mmain(A, tj);
        p = t + (size_t)oi * ld + oj;        // L(bi,bj)(r,c) = U at p[c + r*ld]
    }
}

template <bool SHAPE_T>
__global__ void __launch_bounds__(LL_THREADS, 1)
k_trsv_ll(plasma_desc_t A, int uplo, int backward, Couple C, float *vec,
          unsigned long long *ll, SweepSync *sy, int epoch, plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *Ws = reinterpret_cast<float *>(smem_raw);    // W_u (Wf or Wb), [c*SB + i]
    float *Ms = Ws + LL_SB * LL_SB;                      // M_u
    float *ys = Ms + LL_SB * LL_SB;                      // a block of the solution
    float *ps = ys + LL_SB;                              // b_u - s_u
    float *red = ps + LL_SB;                             // LL_THREADS
    float *red_n = red + LL_THREADS;                     // 16 x SB (shape N)
    __shared__ int blk_s, abort_s;
    // one answer for the whole block: the ticket loop holds barriers
    if (__syncthreads_or(plasma_failed(st))) return;
    const int n = A.m;
    const int nblk = (n + LL_SB - 1) / LL_SB;
    const int tid = threadIdx.x;
    const bool lower = uplo == PlasmaLower;
    if (tid == 0) abort_s = 0;

    for (;;) {
        if (tid == 0) blk_s = atomicAdd(&sy->ticket, 1);
        __syncthreads();
        const int t = blk_s;
        __syncthreads();
        if (t >= nblk) break;
        const int u = backward ? nblk - 1 - t : t;
        const int rows = min(LL_SB, n - u * LL_SB);

        // W_u and M_u to shared memory (read-only factor data)
        const float *wsrc = (backward ? C.Wb : C.Wf) + (size_t)u * LL_SB * LL_SB;
        const float *msrc = (backward ? C.Mb : C.Mf) + (size_t)u * LL_SB * LL_SB;
        for (int e = tid * 4; e < LL_SB * LL_SB; e += LL_THREADS * 4) {
            cp_async_16(Ws + e, wsrc + e, true);
            if (t > 0) cp_async_16(Ms + e, msrc + e, true);
        }
        cp_async_commit();
        float bu = 0.f;
        if (tid < rows) bu = vec[(size_t)u * LL_SB + tid];

        // off the chain: blocks j = 0 .. nnc-1 in sweep order (block
        // k(j) = j forward, nblk-1-j backward), three in flight: the
        // factor elements of block j+3 are requested as soon as block j
        // is consumed
        const int nnc = t > 0 ? t - 1 : 0;
        float acc[8];
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = 0.f;
        bool ok = true;
        if (nnc > 0) {
            float4 b0[8], b1[8], b2[8];
            unsigned long long w0 = 0ull, w1 = 0ull, w2 = 0ull;
            auto blk_of = [&](int j) { return backward ? nblk - 1 - j : j; };
            auto issue = [&](int j, float4 (&b)[8], unsigned long long &w) {
                if (j < nnc) {
                    const int k = blk_of(j);
                    const int kr = min(LL_SB, n - k * LL_SB);
                    const float *p;
                    int ld;
                    row_block_addr<SHAPE_T>(A, lower, backward, u, k, p, ld);
                    if (SHAPE_T) load_t(p, ld, kr, rows, tid, b);
                    else load_n(p, ld, rows, kr, tid, b);
                    w = ll_peek(ll, k, kr, tid);
                }
            };
            auto consume = [&](int j, float4 (&b)[8], unsigned long long &w) -> bool {
                if (j >= nnc) return true;
                const int k = blk_of(j);
                const int kr = min(LL_SB, n - k * LL_SB);
                if (!ll_fetch(ll, sy, k, kr, epoch, ys, tid, &abort_s, w)) return false;
                if (SHAPE_T) fma_t(b, ys, tid, acc);
                else fma_n(b, ys, tid, acc);
                __syncthreads();                    // ys is refilled next
                issue(j + 3, b, w);
                return true;
            };
            issue(0, b0, w0);
            issue(1, b1, w1);
            issue(2, b2, w2);
            for (int j = 0; j < nnc && ok; j += 3) {
                ok = consume(j, b0, w0) && consume(j + 1, b1, w1) && consume(j + 2, b2, w2);
            }
        }
        if (!ok) {
            cp_async_wait<0>();
            if (tid == 0) plasma_fail(st, PlasmaErrorInternal, 0);
            return;
        }
        // s_u in shared memory, then p = b_u - s_u
        if (SHAPE_T) {
            // result column 8w + j summed across the warp; lane j keeps it
            const int lane = tid & 31;
            float mine = 0.f;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                float v = acc[j];
#pragma unroll
                for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                mine = lane == j ? v : mine;
            }
            if (lane < 8) red[8 * (tid >> 5) + lane] = mine;
            __syncthreads();
            if (tid < LL_SB) ps[tid] = tid < rows ? bu - red[tid] : 0.f;
        } else {
            // rows 4(t%32) .. +3, one partial per column group (16 of them):
            // red_n[g][i], summed over g
#pragma unroll
            for (int q = 0; q < 4; q++) red_n[(tid >> 5) * LL_SB + 4 * (tid & 31) + q] = acc[q];
            __syncthreads();
            if (tid < LL_SB) {
                float v = 0.f;
#pragma unroll
                for (int g = 0; g < LL_THREADS / 32; g++) v += red_n[g * LL_SB + tid];
                ps[tid] = tid < rows ? bu - v : 0.f;
            }
        }
        cp_async_wait<0>();
        __syncthreads();
        float y = smem_gemv(Ws, ps, red, tid);      // q_u = W_u p
        if (t > 0) {
            // on the chain: the block just before u in sweep order
            const int kc = backward ? u + 1 : u - 1;
            const int kcr = min(LL_SB, n - kc * LL_SB);
            if (!ll_fetch(ll, sy, kc, kcr, epoch, ys, tid, &abort_s,
                          ll_peek(ll, kc, kcr, tid))) {
                if (tid == 0) plasma_fail(st, PlasmaErrorInternal, 0);
                return;
            }
            y -= smem_gemv(Ms, ys, red, tid);
        }
        if (tid < rows) {
            vec[(size_t)u * LL_SB + tid] = y;
            st_relaxed_u64(ll + (size_t)u * LL_SB + tid, ll_pack(y, epoch));
        }
        __syncthreads();
    }
}

// Per block u of the factor (one CTA per (u, job)): job 0 writes
// Wb_u = Wf_u^T, job 1 Mf_u = Wf_u L(u,u-1) (u >= 1), job 2
// Mb_u = Wf_u^T L(u+1,u)^T (u <= nblk-2); all column-major SB x SB, with
// FP32 products (the coupling keeps the factor's accuracy).
__global__ void __launch_bounds__(256)
k_trsv_couple(plasma_desc_t A, int uplo, float *W, const plasma_devstat_t *st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *Ws = reinterpret_cast<float *>(smem_raw);   // [c][i] stride SB+1
    float *Bs = Ws + LL_SB * (LL_SB + 1);              // [c][j] stride SB+1
    if (plasma_failed(st)) return;
    const int n = A.m, nblk = (n + LL_SB - 1) / LL_SB;
    const int u = blockIdx.x, job = blockIdx.y, tid = threadIdx.x;
    const size_t blk = (size_t)LL_SB * LL_SB;
    const float *Wf = W + (size_t)u * blk;
    float *Wb = W + (size_t)nblk * blk + (size_t)u * blk;
    float *Mf = W + 2 * (size_t)nblk * blk + (size_t)u * blk;
    float *Mb = W + 3 * (size_t)nblk * blk + (size_t)u * blk;
    if (job == 0) {
        for (int e = tid; e < LL_SB * LL_SB; e += 256) {
            const int i = e % LL_SB, c = e / LL_SB;
            Wb[(size_t)c * LL_SB + i] = Wf[(size_t)i * LL_SB + c];
        }
        return;
    }
    const bool fwd = job == 1;
    if ((fwd && u == 0) || (!fwd && u == nblk - 1)) return;
    const bool lower = uplo == PlasmaLower;
    // op(W) with op = identity (forward) or transpose (backward):
    // Ws[c][i] = op(Wf)(i,c)
    for (int e = tid; e < LL_SB * LL_SB; e += 256) {
        const int i = e % LL_SB, c = e / LL_SB;
        Ws[c * (LL_SB + 1) + i] = fwd ? Wf[(size_t)c * LL_SB + i] : Wf[(size_t)i * LL_SB + c];
    }
    // B = L(u,u-1) (forward) or L(u+1,u)^T (backward): Bs[j][c] = B(c,j)
    const int bi = fwd ? u : u + 1, bj = fwd ? u - 1 : u;
    const int ri = min(LL_SB, n - bi * LL_SB), rj = min(LL_SB, n - bj * LL_SB);
    LBlock<float> b = lblock<float, LL_SB>(A, lower, bi, bj);
    for (int e = tid; e < LL_SB * LL_SB; e += 256) {
        const int r = e % LL_SB, c = e / LL_SB;          // L(bi,bj)(r,c)
        const float v = (r < ri && c < rj) ? b.p[(size_t)r * b.si + (size_t)c * b.sj] : 0.f;
        if (fwd) Bs[c * (LL_SB + 1) + r] = v;            // B(r,c): row r of the K index
        else Bs[r * (LL_SB + 1) + c] = v;                // B(c,r) = L(r,c)
    }
    __syncthreads();
    // out(i,j) = sum_c op(W)(i,c) B(c,j); thread (ti,tj) owns 8 x 8
    const int ti = tid & 15, tj = tid >> 4;
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int bb = 0; bb < 8; bb++) acc[a][bb] = 0.f;
    for (int c = 0; c < LL_SB; c++) {
        float wa[8], bv[8];
#pragma unroll
        for (int a = 0; a < 8; a++) wa[a] = Ws[c * (LL_SB + 1) + ti + 16 * a];
#pragma unroll
        for (int bb = 0; bb < 8; bb++) bv[bb] = Bs[(tj + 16 * bb) * (LL_SB + 1) + c];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int bb = 0; bb < 8; bb++) acc[a][bb] += wa[a] * bv[bb];
    }
    float *out = fwd ? Mf : Mb;
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int bb = 0; bb < 8; bb++)
            out[(size_t)(tj + 16 * bb) * LL_SB + ti + 16 * a] = acc[a][bb];
}

constexpr int ll_smem()
{
    return (2 * LL_SB * LL_SB + 2 * LL_SB + LL_THREADS + (LL_THREADS / 32) * LL_SB) * 4;
}
constexpr int couple_smem() { return 2 * LL_SB * (LL_SB + 1) * 4; }

template <typename T, int SB> constexpr int trsv_smem()
{
    return (2 * SB * SB + 3 * SB + TS_THREADS) * (int)sizeof(T);
}

template <typename T, int SB> constexpr int trtri_smem()
{
    return (SB * (SB + 1) + SB * 33) * (int)sizeof(T);
}

template <typename T, int SB>
void launch_trtri(cudaStream_t s, plasma_devstat_t *st, int uplo,
                  const plasma_desc_t &A, void *W, int nblk, int unit = 0)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trtri_blocks<T, SB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trtri_smem<T, SB>());
    }
    k_trtri_blocks<T, SB><<<nblk, 256, trtri_smem<T, SB>(), s>>>(A, uplo, unit, (T *)W, st);
}

template <typename T, int SB>
void launch_trsv(cudaStream_t s, plasma_devstat_t *st, int uplo, int backward,
                 const plasma_desc_t &A, const void *W, void *vec, SweepSync *sy,
                 int epoch, int grid)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsv<T, SB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trsv_smem<T, SB>());
    }
    k_trsv<T, SB><<<grid, TS_THREADS, trsv_smem<T, SB>(), s>>>(
        A, uplo, backward, (const T *)W, (T *)vec, sy, epoch, st);
}

void launch_couple(cudaStream_t s, plasma_devstat_t *st, int uplo, const plasma_desc_t &A,
                   void *W, int nblk)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsv_couple, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             couple_smem());
    }
    k_trsv_couple<<<dim3(nblk, 3), 256, couple_smem(), s>>>(A, uplo, (float *)W, st);
}

template <bool SHAPE_T>
void launch_ll(cudaStream_t s, plasma_devstat_t *st, int uplo, int backward,
               const plasma_desc_t &A, const Couple &C, float *vec, unsigned long long *ll,
               SweepSync *sy, int epoch, int grid)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsv_ll<SHAPE_T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ll_smem());
    }
    k_trsv_ll<SHAPE_T><<<grid, LL_THREADS, ll_smem(), s>>>(A, uplo, backward, C, vec, ll, sy,
                                                           epoch, st);
}

// FP32 factors with 128-row sweep blocks use the coupled sweep (k_trsv_ll)
bool use_ll(const plasma_desc_t &A, int sb)
{
    return A.precision == PlasmaRealFloat && sb == LL_SB;
}

size_t flags_bytes(int nblk)
{
    return (sizeof(int) * (size_t)(nblk + 4) + 255) & ~(size_t)255;
}

}  // namespace

// Sweep block: 128 rows for FP32 factors whose tiles allow it, else 64;
// 0 when the tile size is not a multiple of 64 (no one-launch sweep).
extern "C" int plasma_cuda_trsv_block(plasma_desc_t A)
{
    if (A.mb != A.nb || A.mb % 64 != 0) return 0;
    if (A.precision == PlasmaRealFloat && A.mb % 128 == 0) return 128;
    if (A.precision == PlasmaRealFloat || A.precision == PlasmaRealDouble) return 64;
    return 0;
}

extern "C" size_t plasma_cuda_trsv_sync_bytes(int nblk)
{
    return sizeof(int) * (size_t)(nblk + 4);
}

// Scratch of a sweep: the ready flags, and for the coupled FP32 sweep the
// published solution words (8 bytes per row) after them.
extern "C" size_t plasma_cuda_trsv_scratch_bytes(plasma_desc_t A)
{
    int sb = plasma_cuda_trsv_block(A);
    if (sb == 0) return 0;
    const int nblk = (A.m + sb - 1) / sb;
    size_t b = flags_bytes(nblk);
    if (use_ll(A, sb)) b += (size_t)nblk * sb * sizeof(unsigned long long);
    return b;
}

// Block inverses W (nblk x sb x sb); the coupled FP32 sweep adds W^T and the
// two coupling products (four such arrays).
extern "C" size_t plasma_cuda_trsv_w_bytes(plasma_desc_t A)
{
    int sb = plasma_cuda_trsv_block(A);
    if (sb == 0) return 0;
    size_t nblk = (size_t)(A.m + sb - 1) / sb;
    size_t one = nblk * sb * sb * plasma_element_size(A.precision);
    return use_ll(A, sb) ? 4 * one : one;
}

// Inverses of the SB x SB diagonal blocks of the factor held in A.
extern "C" void plasma_cuda_trtri_blocks(cudaStream_t s, plasma_devstat_t *st,
                                         plasma_enum_t uplo, plasma_desc_t A, void *W)
{
    int sb = plasma_cuda_trsv_block(A);
    if (sb == 0) return;
    int nblk = (A.m + sb - 1) / sb;
    if (nblk == 0) return;
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble)
        launch_trtri<double, 64>(s, st, uplo, A, W, nblk);
    else if (sb == 128)
        launch_trtri<float, 128>(s, st, uplo, A, W, nblk);
    else
        launch_trtri<float, 64>(s, st, uplo, A, W, nblk);
    if (use_ll(A, sb)) {
        PLASMA_COUNT_LAUNCH();
        launch_couple(s, st, uplo, A, W, nblk);
    }
}

// The block inverses for the one-launch sweeps with an LU factor held in
// the general tile matrix A (unit-lower L below the diagonal, U on and
// above it): Wf for L y = b (the sweep with uplo = Lower, forward), Wb for
// U x = y (uplo = Upper, backward: U is the transpose of the logical lower
// factor of upper storage).  Returns 0 (nothing launched) unless the sweep
// block is 64 rows (FP64 tiles, or FP32 tiles whose size is an odd multiple
// of 64).
extern "C" int plasma_cuda_trtri_blocks_lu(cudaStream_t s, plasma_devstat_t *st,
                                           plasma_desc_t A, void *Wf, void *Wb)
{
    const int sb = plasma_cuda_trsv_block(A);
    if (sb != 64) return 0;
    const int nblk = (A.m + sb - 1) / sb;
    if (nblk == 0) return 1;
    PLASMA_COUNT_LAUNCH();
    PLASMA_COUNT_LAUNCH();
    if (A.precision == PlasmaRealDouble) {
        launch_trtri<double, 64>(s, st, PlasmaLower, A, Wf, nblk, 1);
        launch_trtri<double, 64>(s, st, PlasmaUpper, A, Wb, nblk, 0);
    } else {
        launch_trtri<float, 64>(s, st, PlasmaLower, A, Wf, nblk, 1);
        launch_trtri<float, 64>(s, st, PlasmaUpper, A, Wb, nblk, 0);
    }
    return 1;
}

// In-place solve of op(L) x = vec for one right-hand side (vec contiguous):
// backward = 0 solves L y = b, 1 solves L^T x = y, L the logical lower
// Cholesky factor held in A with storage uplo.  W from
// plasma_cuda_trtri_blocks.  sync: device scratch of
// plasma_cuda_trsv_sync_bytes(nblk) bytes, zero-initialised before its
// first use; epoch: distinct non-zero value for every call that reuses it.
extern "C" int plasma_cuda_trsv(cudaStream_t s, plasma_devstat_t *st,
                                plasma_enum_t uplo, int backward,
                                plasma_desc_t A, const void *W, void *vec,
                                void *sync, int epoch, int num_sms)
{
    if (A.mb != A.nb ||
        (A.precision != PlasmaRealDouble && A.precision != PlasmaRealFloat))
        return 0;
    const int sb = plasma_cuda_trsv_block(A);
    if (sb == 0)
        return 0;
    const int nblk = (A.m + sb - 1) / sb;
    if (nblk == 0) return 1;
    SweepSync *sy = (SweepSync *)sync;
    cudaMemsetAsync(&sy->ticket, 0, 2 * sizeof(int), s);
    int grid = nblk < num_sms ? nblk : num_sms;
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    if (use_ll(A, sb)) {
        const size_t one = (size_t)nblk * LL_SB * LL_SB;
        const float *w = (const float *)W;
        Couple C{w, w + one, w + 2 * one, w + 3 * one};
        unsigned long long *ll =
            (unsigned long long *)((char *)sync + flags_bytes(nblk));
        // shape T: forward through upper storage, backward through lower
        const bool shape_t = (uplo == PlasmaLower) == (backward != 0);
        if (shape_t)
            launch_ll<true>(s, st, uplo, backward, A, C, (float *)vec, ll, sy, epoch, grid);
        else
            launch_ll<false>(s, st, uplo, backward, A, C, (float *)vec, ll, sy, epoch, grid);
    } else if (A.precision == PlasmaRealDouble)
        launch_trsv<double, 64>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    else if (sb == 128)
        launch_trsv<float, 128>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    else
        launch_trsv<float, 64>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    double n = A.m, es = plasma_element_size(A.precision);
    plasma_prof_end(prof, s, PLASMA_KCLASS_SOLVE, n * n, es * n * n / 2.0);
    return 1;
}

// In-place solve of op(L) X = B(:, c0 .. c0+ncols-1) for up to 16 columns of
// a tile matrix B (B.i = B.j = 0), the one-launch multi-column sweep
// (k_trsm_rows); W, sync and epoch as for plasma_cuda_trsv.  Returns 0
// (nothing launched) when the factor's tiles admit no block sweep.
extern "C" int plasma_cuda_trsm_rows(cudaStream_t s, plasma_devstat_t *st,
                                     plasma_enum_t uplo, int backward, plasma_desc_t A,
                                     const void *W, plasma_desc_t B, int c0, int ncols,
                                     void *sync, int epoch, int num_sms)
{
    const int sb = plasma_cuda_trsv_block(A);
    if (sb == 0 || B.i != 0 || B.j != 0 || B.precision != A.precision || B.m != A.m ||
        ncols < 1 || ncols > 16 || c0 < 0 || c0 + ncols > B.n)
        return 0;
    const int nblk = (A.m + sb - 1) / sb;
    if (nblk == 0) return 1;
    SweepSync *sy = (SweepSync *)sync;
    cudaMemsetAsync(&sy->ticket, 0, 2 * sizeof(int), s);
    const int grid = nblk < num_sms ? nblk : num_sms;
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    if (A.precision == PlasmaRealDouble) {
        if (ncols <= 4)
            launch_trsm_rows<double, 64, 4>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                            epoch, grid);
        else
            launch_trsm_rows<double, 64, 16>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                             epoch, grid);
    } else if (sb == 128) {
        if (ncols <= 4)
            launch_trsm_rows<float, 128, 4>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                            epoch, grid);
        else
            launch_trsm_rows<float, 128, 16>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                             epoch, grid);
    } else {
        if (ncols <= 4)
            launch_trsm_rows<float, 64, 4>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                           epoch, grid);
        else
            launch_trsm_rows<float, 64, 16>(s, st, uplo, backward, A, W, B, c0, ncols, sy,
                                            epoch, grid);
    }
    double n = A.m, es = plasma_element_size(A.precision);
    plasma_prof_end(prof, s, PLASMA_KCLASS_SOLVE, n * n * ncols,
                    es * (n * n / 2.0 + 2.0 * n * ncols));
    return 1;
}
