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
template <typename T, int SB>
__global__ void __launch_bounds__(256)
k_trtri_blocks(plasma_desc_t A, int uplo, T *W, const plasma_devstat_t *st)
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
        Ls[c * (SB + 1) + i] = (i < rows && c < rows && i >= c)
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
                  const plasma_desc_t &A, void *W, int nblk)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_trtri_blocks<T, SB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trtri_smem<T, SB>());
        attr = true;
    }
    k_trtri_blocks<T, SB><<<nblk, 256, trtri_smem<T, SB>(), s>>>(A, uplo, (T *)W, st);
}

template <typename T, int SB>
void launch_trsv(cudaStream_t s, plasma_devstat_t *st, int uplo, int backward,
                 const plasma_desc_t &A, const void *W, void *vec, SweepSync *sy,
                 int epoch, int grid)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_trsv<T, SB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             trsv_smem<T, SB>());
        attr = true;
    }
    k_trsv<T, SB><<<grid, TS_THREADS, trsv_smem<T, SB>(), s>>>(
        A, uplo, backward, (const T *)W, (T *)vec, sy, epoch, st);
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

extern "C" size_t plasma_cuda_trsv_w_bytes(plasma_desc_t A)
{
    int sb = plasma_cuda_trsv_block(A);
    if (sb == 0) return 0;
    size_t nblk = (size_t)(A.m + sb - 1) / sb;
    return nblk * sb * sb * plasma_element_size(A.precision);
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
    if (A.precision == PlasmaRealDouble)
        launch_trsv<double, 64>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    else if (sb == 128)
        launch_trsv<float, 128>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    else
        launch_trsv<float, 64>(s, st, uplo, backward, A, W, vec, sy, epoch, grid);
    double n = A.m, es = plasma_element_size(A.precision);
    plasma_prof_end(prof, s, PLASMA_KCLASS_SOLVE, n * n, es * n * n / 2.0);
    return 1;
}
