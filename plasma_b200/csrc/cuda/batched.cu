// batched.cu -- thousands of independent SPD systems of uneven size in one
// persistent launch: Cholesky factor (potrf), solve (potrs, one right-hand
// side) and their adjoints.  No reference counterpart (PLASMA factors one
// matrix at a time); the per-matrix algorithm is the reference's blocked
// right-looking Cholesky (compute/pzpotrf.c:37-80 at the scale of one CTA).
//
// Layout: matrix i is column-major n_i x n_i (ld = n_i) at A + off_a[i];
// its right-hand side / solution at B + off_b[i].  A plan (host side) sorts
// the matrices by decreasing size (longest processing time first) and picks
// the block width NB of each size bucket from a measured table.
//
// One CTA per SM, 256 threads, takes the next matrix from an atomic counter
// until the list is exhausted, so large and small matrices balance across
// SMs.  Per matrix, for each block column j0:
//   (a) one warp factors the NB x NB diagonal block, lane r holding row r,
//       pivots broadcast by shuffles (LAPACK's info on a non-positive or NaN
//       pivot, and the matrix is abandoned);
//   (b) every thread solves one row of the panel below, x D^T = a, with D
//       in shared memory; the panel is kept in shared memory;
//   (c) the trailing lower triangle is updated, A22 -= P P^T, by warps on
//       16 x 32 blocks with DMMA (FP64) or the three-product TF32 split
//       (FP32, FP32-accurate), C read (before the products, so the read
//       overlaps them) and written in global memory (L2); the first 32
//       columns first, then warp 0 factors the next diagonal block while
//       the other warps update the rest.
// The solve follows in the same CTA while the factor is in L2: forward by
// block (diagonal block by one warp, the rows below by all threads),
// backward by block (column dot products by warps, then the diagonal block).
#include "common.cuh"
#include "mma.cuh"

#include <stdlib.h>
#include <string.h>

namespace {

constexpr int BT = 256;               // threads per CTA
constexpr int NMAX = 512;             // largest matrix of the batched path
constexpr int NBMAXB = 32;            // largest block width

template <typename T> constexpr int ps_ld() { return NBMAXB + Pad<T>::v; }
// shared memory: panel [NMAX][ps_ld], two 32 x 33 blocks, a vector of NMAX,
// 32 reciprocal pivots, the inverse of the diagonal block [32][ps_ld]
template <typename T> constexpr int batched_smem()
{
    return (NMAX * ps_ld<T>() + 2 * NBMAXB * (NBMAXB + 1) + NMAX + NBMAXB +
            NBMAXB * ps_ld<T>()) * (int)sizeof(T);
}

enum { OP_POSV = 0, OP_POTRF = 1, OP_POTRS = 2, OP_POTRF_ADJ = 3, OP_POTRS_ADJ = 4 };

struct BatchArgs {
    int batch;
    const int *n;               // [batch]
    const long long *off_a;     // [batch] element offsets of the matrices
    const long long *off_b;     // [batch] element offsets of the vectors
    const int *order;           // processing order (largest first)
    const unsigned char *nbsel; // [batch] block width of each matrix (16 or 32)
    void *A;                    // matrices (the factor for solves and adjoints)
    void *B;                    // right-hand sides / solutions (X for the adjoint)
    void *C;                    // Xbar -> Bbar (potrs adjoint)
    void *D;                    // Lbar (adjoints)
    int *info;                  // [batch] (factorisations)
    int *counter;               // zeroed before the launch
    int op;
};

// ------------------------------------------------------------------ factor
// The diagonal block at j0 (jb x jb, lower), factored by one warp,
// right-looking: lane r holds row r in registers (every loop unrolled, so the
// row stays in registers), the block padded to NB x NB with the identity so
// that no step depends on jb.  Per column c: the pivot comes from lane c by
// one shuffle, every lane scales its entry and publishes it in Ds (column c
// at Ds[c * (NBMAXB + 1)]), and the rank-1 update reads the column back as
// broadcast loads, independent of one another.  (Entries above the diagonal
// are updated too, from entries above the diagonal only, and never written
// out.)  The block is read from A, or from Dn (column c at Dn[c * (NBMAXB
// + 1)], its lower triangle) where the update that produced it left a copy.
// Writes L to A and Ds, the reciprocal pivots to rdiag and the first bad
// pivot (LAPACK's info within the block, 0 if none) to *flag.
template <typename T, int NB>
__device__ __forceinline__ void diag_block(T *A, int n, int j0, int jb, T *Ds, T *rdiag,
                                           int *flag, int lane, const T *Dn = nullptr)
{
    constexpr int DL = NBMAXB + 1;
    T v[NB];
#pragma unroll
    for (int c = 0; c < NB; c++)
        v[c] = (lane < jb && c < jb)
                   ? (lane >= c ? (Dn != nullptr ? Dn[c * DL + lane]
                                                 : A[(size_t)(j0 + c) * n + j0 + lane])
                                : T(0))
                   : (lane == c ? T(1) : T(0));
    int bad = 0;
    T myrd = T(1);
#pragma unroll
    for (int c = 0; c < NB; c++) {
        const T d = __shfl_sync(0xffffffffu, v[c], c);
        const bool ok = d > T(0);
        if (!ok && bad == 0 && c < jb) bad = c + 1;
        // one reciprocal square root per pivot: 1/sqrt(d), sqrt(d) = d/sqrt(d)
        const T rd = ok ? rsqrt(d) : T(1);
        if (lane == c) {
            myrd = rd;
            v[c] = ok ? d * rd : T(1);
        } else {
            v[c] *= rd;
        }
        Ds[c * DL + lane] = v[c];
        __syncwarp();
#pragma unroll
        for (int c2 = c + 1; c2 < NB; c2++) v[c2] -= v[c] * Ds[c * DL + c2];
    }
    if (lane < jb) {
#pragma unroll
        for (int c = 0; c < NB; c++)
            if (c < jb && lane >= c) A[(size_t)(j0 + c) * n + j0 + lane] = v[c];
        rdiag[lane] = myrd;
    }
    if (lane == 0) *flag = bad;
}

// The inverse of the factored diagonal block, Li = L^-1 (row i at
// Li[i * ps_ld]), by one warp: lane j solves L y = e_j column by column
// (y_k scaled by its reciprocal pivot, then y_i -= L_ik y_k below it, the
// column of L read from Ds as broadcast loads); every loop unrolled, y kept
// in registers until the end.  Lanes at or beyond NB form zero columns,
// never read.
template <typename T, int NB>
__device__ __forceinline__ void diag_inverse(const T *Ds, const T *rdiag, T *Li, int lane)
{
    constexpr int DL = NBMAXB + 1, LLD = ps_ld<T>();
    T y[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) y[i] = (i == lane) ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k < NB; k++) {
        y[k] *= rdiag[k];
#pragma unroll
        for (int i = k + 1; i < NB; i++) y[i] -= Ds[k * DL + i] * y[k];
    }
#pragma unroll
    for (int i = 0; i < NB; i++) Li[i * LLD + lane] = y[i];
}

// Per block column j0: (b) the panel below the diagonal block, X D^T = A21,
// as the tensor-core product X = A21 D^-T with the inverse formed right
// after the diagonal block was factored (kept in shared memory); (c1) the
// trailing update of the first 32 columns of A22 (they hold the next
// diagonal block and the next panel); then warp 0 factors the next diagonal
// block and inverts it (a) while the other warps finish the trailing update
// (c2), so the single-warp chains of (a) overlap the tensor work.  The trailing update runs on 16 x 32 blocks of
// the lower triangle with DMMA (FP64) or the three-product TF32 split
// (FP32); a warp's block of C is read into registers before its products,
// so the L2 latency of the read overlaps them.  With ys (posv: the
// right-hand side in shared memory) the forward sweep L y = b runs along:
// y_j by warp 0 from the diagonal block while it is in shared memory, the
// rows below from the panel, so the solve afterwards is the backward sweep
// alone.
template <typename T, int SPLIT, int NB>
__device__ int factor_one(T *A, int n, T *Ps, T *Ds, T *rdiag, int *flag, T *ys, T *Li,
                          T *Dn)
{
    constexpr int PLD = ps_ld<T>();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    if (warp == 0) {
        diag_block<T, NB>(A, n, 0, min(NB, n), Ds, rdiag, flag, lane);
        __syncwarp();
        diag_inverse<T, NB>(Ds, rdiag, Li, lane);
    }
    __syncthreads();
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = min(NB, n - j0);
        const int m2 = n - j0 - jb;
        const int bad = *flag;
        if (bad) return j0 + bad;
        // (b) the panel below, X = A21 L_jj^-T: a tensor-core product with
        // the inverse, 16-row blocks taken by the warps in turn (a panel
        // exists only below a full diagonal block, jb = NB), X written to A
        // and to Ps
        {
            T *A21 = A + (size_t)j0 * n + (j0 + jb);
            for (int r0 = warp * 16; r0 < m2; r0 += BT / 2) {
                const int ra = r0 + g;
                T af[NB / 8][4];
#pragma unroll
                for (int k8 = 0; k8 < NB; k8 += 8) {
                    const T *c0 = A21 + (size_t)(k8 + t) * n, *c4 = c0 + (size_t)4 * n;
                    af[k8 / 8][0] = ra < m2 ? c0[ra] : T(0);
                    af[k8 / 8][1] = ra + 8 < m2 ? c0[ra + 8] : T(0);
                    af[k8 / 8][2] = ra < m2 ? c4[ra] : T(0);
                    af[k8 / 8][3] = ra + 8 < m2 ? c4[ra + 8] : T(0);
                }
                T acc[NB / 8][4];
#pragma unroll
                for (int ni = 0; ni < NB / 8; ni++)
#pragma unroll
                    for (int e = 0; e < 4; e++) acc[ni][e] = T(0);
#pragma unroll
                for (int k8 = 0; k8 < NB; k8 += 8)
#pragma unroll
                    for (int ni = 0; ni < NB / 8; ni++) {
                        T bf[2];
                        bf[0] = Li[(ni * 8 + g) * PLD + k8 + t];
                        bf[1] = Li[(ni * 8 + g) * PLD + k8 + t + 4];
                        mma8<SPLIT>(acc[ni], af[k8 / 8], bf);
                    }
#pragma unroll
                for (int ni = 0; ni < NB / 8; ni++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const int r = ra + 8 * h, c = ni * 8 + 2 * t + e;
                            if (r < m2) {
                                A21[(size_t)c * n + r] = acc[ni][2 * h + e];
                                Ps[r * PLD + c] = acc[ni][2 * h + e];
                            }
                        }
            }
        }
        __syncthreads();
        // forward sweep, diagonal block: y_j = L_jj^-1 y_j (warp 0)
        if (ys != nullptr && warp == 0) {
            T y = lane < jb ? ys[j0 + lane] : T(0);
            for (int c = 0; c < jb; c++) {
                if (lane == c) y = y * rdiag[c];
                const T yc = __shfl_sync(0xffffffffu, y, c);
                if (lane > c && lane < jb) y -= Ds[c * (NBMAXB + 1) + lane] * yc;
            }
            if (lane < jb) ys[j0 + lane] = y;
        }
        if (m2 == 0) {
            __syncthreads();
            break;
        }
        const int nrb = (m2 + 15) / 16, ncb = (m2 + 31) / 32;
        T *C = A + (size_t)(j0 + jb) * n + (j0 + jb);   // A22(0,0)
        // blocks (bi, bj) of the lower triangle, bi >= 2 bj, numbered column
        // by column; the warps in [w0, w0 + nw) take the blocks of the block
        // columns [bj0, bj1)
        auto trail = [&](int bj0, int bj1, int w0, int nw) {
            if (warp < w0 || warp >= w0 + nw) return;
            int first = 0, count = 0;
            for (int bj = 0; bj < bj1 && bj < ncb; bj++) {
                const int nb_j = max(0, nrb - 2 * bj);
                if (bj < bj0) first += nb_j;
                else count += nb_j;
            }
            for (int pp = warp - w0; pp < count; pp += nw) {
                int bj = 0, q = first + pp;
                while (q >= nrb - 2 * bj) { q -= nrb - 2 * bj; bj++; }
                const int r0 = (2 * bj + q) * 16, c0 = bj * 32;
                T cv[4][4], acc[4][4];
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const int r = r0 + g + 8 * h, c = c0 + ni * 8 + 2 * t + e;
                            cv[ni][2 * h + e] = (r < m2 && c < m2 && r >= c)
                                                    ? C[(size_t)c * n + r] : T(0);
                            acc[ni][2 * h + e] = T(0);
                        }
#pragma unroll
                for (int k8 = 0; k8 < NB; k8 += 8) {
                    T bf[4][2];
#pragma unroll
                    for (int ni = 0; ni < 4; ni++) {
                        const int cr = c0 + ni * 8 + g;
                        bf[ni][0] = cr < m2 ? Ps[cr * PLD + k8 + t] : T(0);
                        bf[ni][1] = cr < m2 ? Ps[cr * PLD + k8 + t + 4] : T(0);
                    }
                    const int ra = r0 + g;
                    T af[4];
                    af[0] = ra < m2 ? Ps[ra * PLD + k8 + t] : T(0);
                    af[1] = ra + 8 < m2 ? Ps[(ra + 8) * PLD + k8 + t] : T(0);
                    af[2] = ra < m2 ? Ps[ra * PLD + k8 + t + 4] : T(0);
                    af[3] = ra + 8 < m2 ? Ps[(ra + 8) * PLD + k8 + t + 4] : T(0);
#pragma unroll
                    for (int ni = 0; ni < 4; ni++) mma8<SPLIT>(acc[ni], af, bf[ni]);
                }
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const int r = r0 + g + 8 * h, c = c0 + ni * 8 + 2 * t + e;
                            if (r < m2 && c < m2 && r >= c) {
                                const T val = cv[ni][2 * h + e] - acc[ni][2 * h + e];
                                C[(size_t)c * n + r] = val;
                                // the next diagonal block, for (a) to read
                                if (r < NBMAXB) Dn[c * (NBMAXB + 1) + r] = val;
                            }
                        }
            }
        };
        // (c1) the first 32 columns of A22, all warps
        trail(0, 1, 0, BT / 32);
        __syncthreads();
        // (a) the next diagonal block by warp 0, (c2) the rest by the others
        // (after the forward sweep's rows below: y_below -= P y_j)
        if (warp == 0) {
            diag_block<T, NB>(A, n, j0 + jb, min(NB, m2), Ds, rdiag, flag, lane, Dn);
            __syncwarp();
            diag_inverse<T, NB>(Ds, rdiag, Li, lane);
        } else {
            if (ys != nullptr) {
                for (int r = tid - 32; r < m2; r += BT - 32) {
                    T s0 = T(0), s1 = T(0);
#pragma unroll
                    for (int c = 0; c < NB; c += 2) {
                        s0 += Ps[r * PLD + c] * ys[j0 + c];
                        s1 += Ps[r * PLD + c + 1] * ys[j0 + c + 1];
                    }
                    ys[j0 + jb + r] -= s0 + s1;
                }
            }
            trail(1, ncb, 1, BT / 32 - 1);
        }
        __syncthreads();
    }
    return 0;
}

// ------------------------------------------------------------------- solve
// b <- A^-1 b with the factor L in the lower triangle of A (n x n, ld n).
// Each 32 x 32 diagonal block is first staged in shared memory (one parallel
// load), so the warp's substitution reads shared memory only.
template <typename T>
__device__ void solve_one(const T *A, int n, T *b, T *Ys, T *Db, T *Dr, bool forward_done = false)
{
    constexpr int NB = 32, DLD = NB + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!forward_done)
        for (int i = tid; i < n; i += BT) Ys[i] = b[i];
    // forward: L y = b (unless the factorization ran it: Ys holds y)
    for (int j0 = 0; j0 < n && !forward_done; j0 += NB) {
        const int jb = min(NB, n - j0);
        for (int e = tid; e < NB * NB; e += BT) {
            const int r = e % NB, c = e / NB;
            Db[c * DLD + r] = (r < jb && c < jb && r >= c) ? A[(size_t)(j0 + c) * n + j0 + r] : T(0);
        }
        if (tid < jb) Dr[tid] = T(1) / A[(size_t)(j0 + tid) * n + j0 + tid];
        __syncthreads();
        if (warp == 0) {
            T y = lane < jb ? Ys[j0 + lane] : T(0);
            for (int c = 0; c < jb; c++) {
                if (lane == c) y = y * Dr[c];
                const T yc = __shfl_sync(0xffffffffu, y, c);
                if (lane > c && lane < jb) y -= Db[c * DLD + lane] * yc;
            }
            if (lane < jb) Ys[j0 + lane] = y;
        }
        __syncthreads();
        for (int r = j0 + jb + tid; r < n; r += BT) {
            T s = Ys[r];
#pragma unroll 8
            for (int c = 0; c < jb; c++) s -= A[(size_t)(j0 + c) * n + r] * Ys[j0 + c];
            Ys[r] = s;
        }
        __syncthreads();
    }
    // backward: L^T x = y
    for (int j0 = ((n - 1) / NB) * NB; j0 >= 0; j0 -= NB) {
        const int jb = min(NB, n - j0);
        for (int e = tid; e < NB * NB; e += BT) {
            const int r = e % NB, c = e / NB;
            Db[c * DLD + r] = (r < jb && c < jb && r >= c) ? A[(size_t)(j0 + c) * n + j0 + r] : T(0);
        }
        if (tid < jb) Dr[tid] = T(1) / A[(size_t)(j0 + tid) * n + j0 + tid];
        for (int c = warp; c < jb; c += BT / 32) {
            T s = T(0);
            for (int i = j0 + jb + lane; i < n; i += 32) s += A[(size_t)(j0 + c) * n + i] * Ys[i];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (lane == 0) Ys[j0 + c] -= s;
        }
        __syncthreads();
        if (warp == 0) {
            T x = lane < jb ? Ys[j0 + lane] : T(0);
            for (int c = jb - 1; c >= 0; c--) {
                if (lane == c) x = x * Dr[c];
                const T xc = __shfl_sync(0xffffffffu, x, c);
                if (lane < c) x -= Db[lane * DLD + c] * xc;
            }
            if (lane < jb) Ys[j0 + lane] = x;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += BT) b[i] = Ys[i];
    __syncthreads();
}

// ------------------------------------------------------------ potrs adjoint
// xbar <- A^-1 xbar (= bbar); Lbar -= tril(bbar (L^T x)^T + x (L^T bbar)^T)
template <typename T>
__device__ void solve_adjoint_one(const T *Lf, int n, const T *x, T *xbar, T *Lbar, T *Ys,
                                  T *U, T *Db, T *Dr)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    solve_one<T>(Lf, n, xbar, Ys, Db, Dr);         // Ys keeps bbar
    T *u1 = U, *u2 = U + NMAX;                     // L^T x, L^T bbar
    for (int c = warp; c < n; c += BT / 32) {
        T s1 = T(0), s2 = T(0);
        for (int r = c + lane; r < n; r += 32) {
            const T l = Lf[(size_t)c * n + r];
            s1 += l * x[r];
            s2 += l * Ys[r];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, off);
            s2 += __shfl_xor_sync(0xffffffffu, s2, off);
        }
        if (lane == 0) { u1[c] = s1; u2[c] = s2; }
    }
    __syncthreads();
    for (int c = warp; c < n; c += BT / 32)
        for (int r = c + lane; r < n; r += 32)
            Lbar[(size_t)c * n + r] -= Ys[r] * u1[c] + x[r] * u2[c];
    __syncthreads();
}

// ------------------------------------------------------------ potrf adjoint
// Blocked reverse mode of the Cholesky factor, walking block columns from the
// last to the first and recomputing from the factor L (lower triangle of Lf):
//   Cbar <- Cbar D^-1;  Bbar -= Cbar R;  Dbar <- tril(Dbar) - tril(Cbar^T C);
//   Dbar <- unblocked reverse of the diagonal block;
//   Rbar -= Cbar^T B + (Dbar + Dbar^T) R
// (R, D, B, C: the blocks left of, on, below-left of and below the diagonal
// block; bars the same blocks of Lbar).  The result Abar is lower triangular
// and the symmetric cotangent is (Abar + Abar^T)/2 with Abar's own diagonal,
// written into both triangles of Lbar at the end.
template <typename T>
__device__ void factor_adjoint_one(const T *Lf, int n, T *Lb, T *Cs, T *Ds, T *Dbs)
{
    constexpr int NB = 32, CLD = NB + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = n; k > 0; k -= NB) {
        const int j = max(0, k - NB), jb = k - j, m2 = n - k;
        for (int e = tid; e < NB * NB; e += BT) {
            const int r = e % NB, c = e / NB;
            const bool in = r < jb && c < jb && r >= c;
            Ds[c * CLD + r] = in ? Lf[(size_t)(j + c) * n + j + r] : T(0);
            Dbs[c * CLD + r] = in ? Lb[(size_t)(j + c) * n + j + r] : T(0);
        }
        __syncthreads();
        // (1) Cbar <- Cbar D^-1, one thread per row
        for (int r = tid; r < m2; r += BT) {
            T x[NB];
#pragma unroll
            for (int c = 0; c < NB; c++) x[c] = c < jb ? Lb[(size_t)(j + c) * n + k + r] : T(0);
#pragma unroll
            for (int c = NB - 1; c >= 0; c--) {
                if (c < jb) {
                    T s = x[c];
#pragma unroll
                    for (int c2 = c + 1; c2 < NB; c2++)
                        if (c2 < jb) s -= x[c2] * Ds[c * CLD + c2];
                    x[c] = s / Ds[c * CLD + c];
                }
            }
#pragma unroll
            for (int c = 0; c < NB; c++) {
                if (c < jb) Lb[(size_t)(j + c) * n + k + r] = x[c];
                Cs[r * CLD + c] = x[c];
            }
        }
        __syncthreads();
        // (2) Bbar -= Cbar R   (rows k.., columns 0..j)
        for (int e = tid; e < m2 * j; e += BT) {
            const int r = e % m2, col = e / m2;
            const T *Rc = Lf + (size_t)col * n + j;
            T s = T(0);
            for (int c = 0; c < jb; c++) s += Cs[r * CLD + c] * Rc[c];
            Lb[(size_t)col * n + k + r] -= s;
        }
        // (3) Dbar -= tril(Cbar^T C)
        for (int e = tid; e < jb * jb; e += BT) {
            const int i = e % jb, c = e / jb;
            if (i < c) continue;
            const T *Cc = Lf + (size_t)(j + c) * n + k;
            T s = T(0);
            for (int r = 0; r < m2; r++) s += Cs[r * CLD + i] * Cc[r];
            Dbs[c * CLD + i] -= s;
        }
        __syncthreads();
        // (4) unblocked reverse on the diagonal block, one warp, lane = column
        if (warp == 0) {
            for (int jj = jb - 1; jj >= 0; jj--) {
                const T djj = Ds[jj * CLD + jj];
                T p = (lane > jj && lane < jb) ? Ds[jj * CLD + lane] * Dbs[jj * CLD + lane] : T(0);
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) p += __shfl_xor_sync(0xffffffffu, p, off);
                if (lane == 0) Dbs[jj * CLD + jj] -= p / djj;
                __syncwarp();
                if (lane >= jj && lane < jb) Dbs[jj * CLD + lane] /= djj;
                __syncwarp();
                if (lane < jj) {
                    T s = T(0);
                    for (int r = jj; r < jb; r++) s += Dbs[jj * CLD + r] * Ds[lane * CLD + r];
                    Dbs[lane * CLD + jj] -= s;
                    const T ljc = Ds[lane * CLD + jj];
                    for (int r = jj + 1; r < jb; r++) Dbs[lane * CLD + r] -= Dbs[jj * CLD + r] * ljc;
                }
                __syncwarp();
                if (lane == 0) Dbs[jj * CLD + jj] *= T(0.5);
                __syncwarp();
            }
        }
        __syncthreads();
        // (5) Rbar -= Cbar^T B + (Dbar + Dbar^T) R   (rows j..k, columns 0..j)
        for (int e = tid; e < jb * j; e += BT) {
            const int i = e % jb, col = e / jb;
            const T *Bc = Lf + (size_t)col * n + k;
            const T *Rc = Lf + (size_t)col * n + j;
            T s = T(0);
            for (int r = 0; r < m2; r++) s += Cs[r * CLD + i] * Bc[r];
            for (int c = 0; c < jb; c++)
                s += (Dbs[c * CLD + i] + Dbs[i * CLD + c]) * Rc[c];
            Lb[(size_t)col * n + j + i] -= s;
        }
        for (int e = tid; e < jb * jb; e += BT) {
            const int r = e % jb, c = e / jb;
            if (r >= c) Lb[(size_t)(j + c) * n + j + r] = Dbs[c * CLD + r];
        }
        __syncthreads();
    }
    // symmetric cotangent in both triangles
    for (size_t e = tid; e < (size_t)n * n; e += BT) {
        const int r = (int)(e % n), c = (int)(e / n);
        if (r > c) {
            const T v = T(0.5) * Lb[(size_t)c * n + r];
            Lb[(size_t)c * n + r] = v;
            Lb[(size_t)r * n + c] = v;
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------ kernel
template <typename T, int SPLIT>
__global__ void __launch_bounds__(BT, 1)
k_batched(BatchArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Ps = reinterpret_cast<T *>(smem_raw);        // [NMAX][ps_ld]
    T *Ds = Ps + NMAX * ps_ld<T>();                 // [32][33]
    T *D2 = Ds + NBMAXB * (NBMAXB + 1);             // [32][33]
    T *Ys = D2 + NBMAXB * (NBMAXB + 1);             // [NMAX]
    T *rdiag = Ys + NMAX;                           // [32]
    T *Li = rdiag + NBMAXB;                         // [32][ps_ld] diagonal block inverse
    __shared__ int idx_s, flag_s;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) idx_s = atomicAdd(a.counter, 1);
        __syncthreads();
        const int idx = idx_s;
        __syncthreads();
        if (idx >= a.batch) break;
        const int m = a.order[idx];
        const int n = a.n[m];
        T *A = (T *)a.A + a.off_a[m];
        if (a.op == OP_POSV || a.op == OP_POTRF) {
            T *b = (T *)a.B + a.off_b[m];
            T *ys = nullptr;
            if (a.op == OP_POSV) {
                for (int i = tid; i < n; i += BT) Ys[i] = b[i];
                __syncthreads();
                ys = Ys;
            }
            const int info = a.nbsel[m] == 16
                                 ? factor_one<T, SPLIT, 16>(A, n, Ps, Ds, rdiag, &flag_s, ys, Li, D2)
                                 : factor_one<T, SPLIT, 32>(A, n, Ps, Ds, rdiag, &flag_s, ys, Li, D2);
            if (tid == 0) a.info[m] = info;
            __syncthreads();
            if (info == 0 && a.op == OP_POSV) solve_one<T>(A, n, b, Ys, D2, rdiag, true);
        } else if (a.op == OP_POTRS) {
            solve_one<T>(A, n, (T *)a.B + a.off_b[m], Ys, D2, rdiag);
        } else if (a.op == OP_POTRS_ADJ) {
            solve_adjoint_one<T>(A, n, (const T *)a.B + a.off_b[m], (T *)a.C + a.off_b[m],
                                 (T *)a.D + a.off_a[m], Ys, Ps, D2, rdiag);
        } else {
            factor_adjoint_one<T>(A, n, (T *)a.D + a.off_a[m], Ps, Ds, D2);
        }
    }
}

template <typename T, int SPLIT>
void launch_batched(cudaStream_t s, const BatchArgs &a, int grid)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_batched<T, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             batched_smem<T>());
    }
    k_batched<T, SPLIT><<<grid, BT, batched_smem<T>(), s>>>(a);
}

}  // namespace

// ------------------------------------------------------------------- plans
struct plasma_batch_s {
    int batch;
    int precision;
    int *d_n;
    long long *d_off_a, *d_off_b;
    int *d_order;
    unsigned char *d_nbsel;
    int *d_counter;
    long long *h_off_a, *h_off_b;
    long long elems_a, elems_b;
    int device;
    int graph;                  // replay launches from cached CUDA graphs
    cudaGraphExec_t exec[5];    // one per operation
    void *g_ptr[5][5];          // the pointers each graph was captured with
};

static void batch_free(plasma_batch_t *p)
{
    if (p == NULL) return;
    for (int i = 0; i < 5; i++)
        if (p->exec[i]) cudaGraphExecDestroy(p->exec[i]);
    cudaFree(p->d_n);
    cudaFree(p->d_off_a);
    cudaFree(p->d_off_b);
    cudaFree(p->d_order);
    cudaFree(p->d_nbsel);
    cudaFree(p->d_counter);
    free(p->h_off_a);
    free(p->h_off_b);
    free(p);
}

extern "C" int plasma_batch_create(plasma_enum_t precision, int batch, const int *n,
                                   plasma_batch_t **plan)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) return PlasmaErrorNotInitialized;
    if (precision != PlasmaRealDouble && precision != PlasmaRealFloat) return -1;
    if (batch < 0) return -2;
    if (n == NULL && batch > 0) return -3;
    if (plan == NULL) return -4;
    for (int i = 0; i < batch; i++)
        if (n[i] < 0 || n[i] > NMAX) {
            plasma_error("plasma_batch_create: matrix orders must lie in [0, 512]");
            return -3;
        }
    if (plasma->device < 0) return PlasmaErrorEnvironment;
    plasma_batch_t *p = (plasma_batch_t *)calloc(1, sizeof(plasma_batch_t));
    if (p == NULL) return PlasmaErrorOutOfMemory;
    p->batch = batch;
    p->precision = precision;
    p->device = plasma->device;
    const int cnt = batch > 0 ? batch : 1;
    p->h_off_a = (long long *)malloc(sizeof(long long) * cnt);
    p->h_off_b = (long long *)malloc(sizeof(long long) * cnt);
    int *order = (int *)malloc(sizeof(int) * cnt);
    unsigned char *nbsel = (unsigned char *)malloc(cnt);
    if (!p->h_off_a || !p->h_off_b || !order || !nbsel) {
        free(order); free(nbsel); batch_free(p);
        return PlasmaErrorOutOfMemory;
    }
    // packed column-major matrices and vectors, each start 32-element aligned
    long long oa = 0, ob = 0;
    for (int i = 0; i < batch; i++) {
        p->h_off_a[i] = oa;
        p->h_off_b[i] = ob;
        oa += ((long long)n[i] * n[i] + 31) / 32 * 32;
        ob += ((long long)n[i] + 31) / 32 * 32;
        order[i] = i;
        nbsel[i] = (unsigned char)plasma_tuning_get_batched_nb(precision, n[i]);
    }
    p->elems_a = oa;
    p->elems_b = ob;
    // longest processing time first: decreasing n (stable)
    int *tmp = (int *)malloc(sizeof(int) * cnt);
    if (tmp == NULL) {
        free(order); free(nbsel); batch_free(p);
        return PlasmaErrorOutOfMemory;
    }
    {
        // counting sort by n, largest first
        int hist[NMAX + 2] = {0};
        for (int i = 0; i < batch; i++) hist[NMAX - n[i]]++;
        int acc = 0;
        for (int v = 0; v <= NMAX + 1; v++) { int c = hist[v]; hist[v] = acc; acc += c; }
        for (int i = 0; i < batch; i++) tmp[hist[NMAX - n[i]]++] = i;
        memcpy(order, tmp, sizeof(int) * cnt);
    }
    free(tmp);
    bool ok = cudaMalloc(&p->d_n, sizeof(int) * cnt) == cudaSuccess &&
              cudaMalloc(&p->d_off_a, sizeof(long long) * cnt) == cudaSuccess &&
              cudaMalloc(&p->d_off_b, sizeof(long long) * cnt) == cudaSuccess &&
              cudaMalloc(&p->d_order, sizeof(int) * cnt) == cudaSuccess &&
              cudaMalloc(&p->d_nbsel, cnt) == cudaSuccess &&
              cudaMalloc(&p->d_counter, sizeof(int)) == cudaSuccess;
    if (ok && batch > 0) {
        ok = cudaMemcpy(p->d_n, n, sizeof(int) * batch, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_off_a, p->h_off_a, sizeof(long long) * batch,
                        cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_off_b, p->h_off_b, sizeof(long long) * batch,
                        cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_order, order, sizeof(int) * batch, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             cudaMemcpy(p->d_nbsel, nbsel, batch, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    free(order);
    free(nbsel);
    if (!ok) {
        cudaGetLastError();
        batch_free(p);
        return PlasmaErrorOutOfMemory;
    }
    *plan = p;
    return PlasmaSuccess;
}

extern "C" void plasma_batch_destroy(plasma_batch_t *plan)
{
    if (plan) cudaDeviceSynchronize();
    batch_free(plan);
}

extern "C" long long plasma_batch_matrix_elems(const plasma_batch_t *plan)
{
    return plan ? plan->elems_a : 0;
}

extern "C" long long plasma_batch_vector_elems(const plasma_batch_t *plan)
{
    return plan ? plan->elems_b : 0;
}

extern "C" int plasma_batch_offsets(const plasma_batch_t *plan, long long *off_a,
                                    long long *off_b)
{
    if (plan == NULL) return -1;
    if (off_a) memcpy(off_a, plan->h_off_a, sizeof(long long) * plan->batch);
    if (off_b) memcpy(off_b, plan->h_off_b, sizeof(long long) * plan->batch);
    return PlasmaSuccess;
}

extern "C" int plasma_batch_set_graph(plasma_batch_t *plan, int on)
{
    if (plan == NULL) return -1;
    plan->graph = on != 0;
    return PlasmaSuccess;
}

// One batched operation: the counter reset and one persistent launch on the
// context stream, or the replay of the CUDA graph that holds both.
static int batch_run(plasma_batch_t *p, int prec, int op, void *A, void *B, void *C, void *D,
                     int *info)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) return PlasmaErrorNotInitialized;
    if (p == NULL) return -1;
    if (p->precision != prec) {
        plasma_error("batched call: precision differs from the plan's");
        return -1;
    }
    if (p->batch == 0) return PlasmaSuccess;
    if (A == NULL || ((op == OP_POSV || op == OP_POTRF) && info == NULL) ||
        ((op == OP_POSV || op == OP_POTRS || op == OP_POTRS_ADJ) && B == NULL) ||
        (op == OP_POTRS_ADJ && C == NULL) ||
        ((op == OP_POTRF_ADJ || op == OP_POTRS_ADJ) && D == NULL))
        return -2;
    BatchArgs a;
    a.batch = p->batch;
    a.n = p->d_n;
    a.off_a = p->d_off_a;
    a.off_b = p->d_off_b;
    a.order = p->d_order;
    a.nbsel = p->d_nbsel;
    a.A = A;
    a.B = B;
    a.C = C;
    a.D = D;
    a.info = info;
    a.counter = p->d_counter;
    a.op = op;
    int grid = plasma->num_sms;          // one CTA per SM (registers, shared memory)
    if (grid > p->batch) grid = p->batch;
    cudaStream_t s = plasma->stream;

    void *key[5] = {A, B, C, D, (void *)info};
    if (p->graph) {
        if (p->exec[op] == NULL || memcmp(p->g_ptr[op], key, sizeof(key)) != 0) {
            if (p->exec[op]) {
                cudaGraphExecDestroy(p->exec[op]);
                p->exec[op] = NULL;
            }
            cudaStream_t cap;
            if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
                return PlasmaErrorEnvironment;
            cudaGraph_t g = NULL;
            cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            cudaMemsetAsync(p->d_counter, 0, sizeof(int), cap);
            if (prec == PlasmaRealDouble) launch_batched<double, 1>(cap, a, grid);
            else launch_batched<float, 3>(cap, a, grid);
            cudaError_t rc = cudaStreamEndCapture(cap, &g);
            if (rc == cudaSuccess)
                rc = cudaGraphInstantiate(&p->exec[op], g, 0);
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            if (rc != cudaSuccess) {
                cudaGetLastError();
                p->exec[op] = NULL;
                return PlasmaErrorEnvironment;
            }
            memcpy(p->g_ptr[op], key, sizeof(key));
        }
        PLASMA_COUNT_LAUNCH();
        return cudaGraphLaunch(p->exec[op], s) == cudaSuccess ? PlasmaSuccess
                                                               : PlasmaErrorEnvironment;
    }
    cudaMemsetAsync(p->d_counter, 0, sizeof(int), s);
    PLASMA_COUNT_LAUNCH();
    if (prec == PlasmaRealDouble) launch_batched<double, 1>(s, a, grid);
    else launch_batched<float, 3>(s, a, grid);
    return PlasmaSuccess;
}

extern "C" int plasma_dposv_batched(plasma_batch_t *plan, double *A, double *B, int *info)
{ return batch_run(plan, PlasmaRealDouble, OP_POSV, A, B, NULL, NULL, info); }
extern "C" int plasma_sposv_batched(plasma_batch_t *plan, float *A, float *B, int *info)
{ return batch_run(plan, PlasmaRealFloat, OP_POSV, A, B, NULL, NULL, info); }
extern "C" int plasma_dpotrf_batched(plasma_batch_t *plan, double *A, int *info)
{ return batch_run(plan, PlasmaRealDouble, OP_POTRF, A, NULL, NULL, NULL, info); }
extern "C" int plasma_spotrf_batched(plasma_batch_t *plan, float *A, int *info)
{ return batch_run(plan, PlasmaRealFloat, OP_POTRF, A, NULL, NULL, NULL, info); }
extern "C" int plasma_dpotrs_batched(plasma_batch_t *plan, const double *L, double *B)
{ return batch_run(plan, PlasmaRealDouble, OP_POTRS, (void *)L, B, NULL, NULL, NULL); }
extern "C" int plasma_spotrs_batched(plasma_batch_t *plan, const float *L, float *B)
{ return batch_run(plan, PlasmaRealFloat, OP_POTRS, (void *)L, B, NULL, NULL, NULL); }
extern "C" int plasma_dpotrf_adjoint_batched(plasma_batch_t *plan, const double *L,
                                             double *Lbar)
{ return batch_run(plan, PlasmaRealDouble, OP_POTRF_ADJ, (void *)L, NULL, NULL, Lbar, NULL); }
extern "C" int plasma_spotrf_adjoint_batched(plasma_batch_t *plan, const float *L,
                                             float *Lbar)
{ return batch_run(plan, PlasmaRealFloat, OP_POTRF_ADJ, (void *)L, NULL, NULL, Lbar, NULL); }
extern "C" int plasma_dpotrs_adjoint_batched(plasma_batch_t *plan, const double *L,
                                             const double *X, double *Xbar, double *Lbar)
{ return batch_run(plan, PlasmaRealDouble, OP_POTRS_ADJ, (void *)L, (void *)X, Xbar, Lbar, NULL); }
extern "C" int plasma_spotrs_adjoint_batched(plasma_batch_t *plan, const float *L,
                                             const float *X, float *Xbar, float *Lbar)
{ return batch_run(plan, PlasmaRealFloat, OP_POTRS_ADJ, (void *)L, (void *)X, Xbar, Lbar, NULL); }
