// potrf_smem.cu -- FP32 diagonal-tile Cholesky with the whole tile in shared
// memory (plasma_core_spotrf on A(k,k), compute/pzpotrf.c:41-44, the first
// step of every column of the tile factorization and so the head of the
// critical path).
//
// The lower triangle of an nk x nk tile (nk a multiple of 32, <= 256) is
// held in shared memory packed by 32-column blocks: block column j keeps
// rows 32j .. nk-1 column-major with leading dimension nk - 32j + 8 (a
// multiple of 8, so that every 4-row piece is a 16-byte load): 156 KB for
// nk = 256.  One CTA of 16 warps walks the block columns right-looking, in
// FP32 arithmetic (the reference's spotrf is FP32 too):
//   (a) one warp factors the 32 x 32 diagonal block, lane r holding row r,
//       pivots broadcast by shuffles, LAPACK's info on a non-positive pivot;
//   (b) a thread per row below solves x D^T = a by substitution;
//   (c) the warps share the trailing lower triangle in 32 x 32 blocks,
//       C -= X X^T, register-blocked FMAs on 16-byte shared-memory loads
//       (each lane four rows by eight columns, 32 FMAs per three loads).  Global
// memory is touched twice: one cp.async load of the tile and one store of
// the factor.
#include "common.cuh"

namespace {

constexpr int SM_THREADS = 512;
constexpr int SM_NBMAX = 256;
constexpr int SM_PAD = 8;

__host__ __device__ constexpr int col_ld(int nk, int j) { return nk - 32 * j + SM_PAD; }
__host__ __device__ constexpr int col_off(int nk, int j)
{
    // sum over i < j of 32 * (nk - 32 i + PAD)
    return 32 * (j * (nk + SM_PAD) - 32 * (j * (j - 1) / 2));
}
constexpr int smem_floats(int nk) { return col_off(nk, nk / 32); }

// One 32 x 32 product step on shared-memory operands for a warp:
// acc[a][b] += sum_k Xa(r0 + a, k) Xb(c0 + b, k), r0 = 4 (lane & 7),
// c0 = 8 (lane >> 3), Xa(r, k) = xa[k*lda + r], Xb(c, k) = xb[k*ldb + c]
// (16-byte loads: four rows, eight columns; 32 FMAs per 3 loads).
__device__ __forceinline__ void warp_block_32(const float *xa, int lda, const float *xb,
                                              int ldb, float (&acc)[4][8], int lane)
{
    const int r0 = 4 * (lane & 7), c0 = 8 * (lane >> 3);
#pragma unroll 4
    for (int kk = 0; kk < 32; kk++) {
        const float4 a = *reinterpret_cast<const float4 *>(xa + kk * lda + r0);
        const float4 b0 = *reinterpret_cast<const float4 *>(xb + kk * ldb + c0);
        const float4 b1 = *reinterpret_cast<const float4 *>(xb + kk * ldb + c0 + 4);
        const float av[4] = {a.x, a.y, a.z, a.w};
        const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int q = 0; q < 8; q++) acc[i][q] += av[i] * bv[q];
    }
}

__global__ void __launch_bounds__(SM_THREADS, 1)
k_potrf_diag_smem(plasma_desc_t A, int k, int iinfo, plasma_devstat_t *st, int call)
{
    extern __shared__ __align__(16) float S[];
    __shared__ float rdiag[32];
    __shared__ int flag;
    if (plasma_failed(st)) return;
    float *T = (float *)plasma_tile_addr(A, k, k);
    const int ldt = plasma_tile_mmain(A, k);
    const int nk = plasma_tile_mview(A, k);
    const int nbc = nk / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // load the lower triangle by block columns, 16-byte copies
    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        for (int cc = warp; cc < 32; cc += SM_THREADS / 32)
            for (int q = lane; q < R / 4; q += 32)
                cp_async_16(S + off + cc * ld + 4 * q,
                            T + (size_t)(32 * j + cc) * ldt + 32 * j + 4 * q, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        float *P = S + off;                        // block column j, P[cc*ld + rr]
        // (a) the diagonal block, one warp, lane r holding row r; the pivot's
        //     reciprocal square root is one special-function operation on
        //     the chain (L(c,c) = d rsqrt(d))
        if (warp == 0) {
            float v[32];
#pragma unroll
            for (int c = 0; c < 32; c++) v[c] = lane >= c ? P[c * ld + lane] : 0.f;
            int bad = 0;
            float myrd = 1.f;
#pragma unroll
            for (int c = 0; c < 32; c++) {
                const float d = __shfl_sync(0xffffffffu, v[c], c);
                const bool ok = d > 0.f;
                if (!ok && bad == 0) bad = c + 1;
                const float rd = ok ? rsqrtf(d) : 1.f;
                if (lane == c) myrd = rd;
                if (lane >= c) v[c] = lane == c ? (ok ? d * rd : 1.f) : v[c] * rd;
                // a fixed trip count keeps v[] in registers (full unroll)
#pragma unroll
                for (int c2 = 0; c2 < 32; c2++) {
                    if (c2 > c) {
                        const float l = __shfl_sync(0xffffffffu, v[c], c2);
                        if (lane >= c2) v[c2] -= v[c] * l;
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < 32; c++)
                if (lane >= c) P[c * ld + lane] = v[c];
            rdiag[lane] = myrd;
            if (lane == 0) flag = bad;
        }
        __syncthreads();
        if (flag) {
            if (tid == 0) plasma_fail(st, iinfo + 32 * j + flag, call);
            return;
        }
        // (b) rows below: x D^T = a, a thread per row, column-oriented
        //     substitution (x_c final, then its multiple of column c of the
        //     block leaves the later entries); column c of the block read
        //     as 16-byte pieces (144 loads per row instead of 528)
        for (int rr = 32 + tid; rr < R; rr += SM_THREADS) {
            float x[32];
#pragma unroll
            for (int c = 0; c < 32; c++) x[c] = P[c * ld + rr];
#pragma unroll
            for (int c = 0; c < 32; c++) {
                x[c] *= rdiag[c];
#pragma unroll
                for (int q = (c + 1) / 4; q < 8; q++) {
                    const float4 l = *reinterpret_cast<const float4 *>(P + c * ld + 4 * q);
                    if (4 * q + 0 > c) x[4 * q + 0] -= x[c] * l.x;
                    if (4 * q + 1 > c) x[4 * q + 1] -= x[c] * l.y;
                    if (4 * q + 2 > c) x[4 * q + 2] -= x[c] * l.z;
                    if (4 * q + 3 > c) x[4 * q + 3] -= x[c] * l.w;
                }
            }
#pragma unroll
            for (int c = 0; c < 32; c++) P[c * ld + rr] = x[c];
        }
        __syncthreads();
        // (c) trailing lower triangle: block columns j+1 .. nbc-1 in 32 x 32
        //     blocks, C -= X X^T
        const int m = nbc - j - 1;
        const int npairs = m * (m + 1) / 2;
        for (int p = warp; p < npairs; p += SM_THREADS / 32) {
            int bj = 0, q = p;
            while (q >= m - bj) { q -= m - bj; bj++; }
            const int bi = bj + q;
            const int jc = j + 1 + bj;                       // block column of C
            float *C = S + col_off(nk, jc) + 32 * (bi - bj);  // C(i, c) = C[c*ldc + i]
            const int ldc = col_ld(nk, jc);
            float acc[4][8];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 8; b++) acc[a][b] = 0.f;
            warp_block_32(P + 32 * (1 + bi), ld, P + 32 * (1 + bj), ld, acc, lane);
            const int r0 = 4 * (lane & 7), c0 = 8 * (lane >> 3);
            if (bi != bj) {
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    float4 *cp = reinterpret_cast<float4 *>(C + (c0 + b) * ldc + r0);
                    float4 cv = *cp;
                    cv.x -= acc[0][b]; cv.y -= acc[1][b]; cv.z -= acc[2][b]; cv.w -= acc[3][b];
                    *cp = cv;
                }
            } else {
#pragma unroll
                for (int b = 0; b < 8; b++)
#pragma unroll
                    for (int a = 0; a < 4; a++)
                        if (r0 + a >= c0 + b) C[(c0 + b) * ldc + r0 + a] -= acc[a][b];
            }
        }
        __syncthreads();
    }
    // store the factor (lower triangle): 16-byte stores below the diagonal
    // block of each column, element stores of its lower part in the block
    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        for (int cc = warp; cc < 32; cc += SM_THREADS / 32) {
            float *tc = T + (size_t)(32 * j + cc) * ldt + 32 * j;
            const float *sc = S + off + cc * ld;
            for (int q = 8 + lane; q < R / 4; q += 32)
                *reinterpret_cast<float4 *>(tc + 4 * q) =
                    *reinterpret_cast<const float4 *>(sc + 4 * q);
            if (lane >= cc) tc[lane] = sc[lane];
        }
    }
}

void launch(cudaStream_t s, plasma_devstat_t *st, int call, const plasma_desc_t &A, int k,
            int iinfo, int bytes)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_potrf_diag_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem_floats(SM_NBMAX) * 4);
    }
    k_potrf_diag_smem<<<1, SM_THREADS, bytes, s>>>(A, k, iinfo, st, call);
}

}  // namespace

// FP32 lower tiles whose order is a multiple of 32 (at most 256) with a
// 16-byte aligned leading dimension; returns 0 (nothing launched) otherwise.
extern "C" int plasma_cuda_potrf_diag_smem(cudaStream_t s, plasma_devstat_t *st, int call,
                                           plasma_enum_t uplo, plasma_desc_t A, int k,
                                           int iinfo, int split)
{
    const int nk = plasma_tile_mview(A, k);
    if (uplo != PlasmaLower || A.precision != PlasmaRealFloat || A.mb != A.nb ||
        nk % 32 != 0 || nk > SM_NBMAX || nk == 0 || plasma_tile_mmain(A, k) % 4 != 0 ||
        ((uintptr_t)plasma_tile_addr(A, k, k) & 15) != 0)
        return 0;
    (void)split;                  // FP32 arithmetic whatever the update's products
    launch(s, st, call, A, k, iinfo, smem_floats(nk) * 4);
    return 1;
}
