// potrf_smem.cu -- FP32 diagonal-tile Cholesky with the whole tile in shared
// memory (plasma_core_spotrf on A(k,k), compute/pzpotrf.c:41-44, the first
// step of every column of the tile factorization and so the head of the
// critical path).
//
// The lower triangle of an nk x nk tile (nk a multiple of 32, <= 256) is
// held in shared memory packed by 32-column blocks: block column j keeps
// rows 32j .. nk-1 column-major with leading dimension nk - 32j + 8 (the
// +8 makes the tensor-core fragment loads conflict-free): 156 KB for
// nk = 256.  One CTA of 16 warps walks the block columns right-looking:
//   (a) one warp factors the 32 x 32 diagonal block, lane r holding row r,
//       pivots broadcast by shuffles, LAPACK's info on a non-positive pivot;
//   (b) one thread per row below solves x D^T = a against the block;
//   (c) the warps share the trailing lower triangle in 32 x 32 blocks,
//       C -= X X^T with TF32 mma.sync, three products per FP32 product
//       (SPLIT = 3: FP32-accurate) or one (SPLIT = 1, the TF32/BF16 modes).
// Global memory is touched twice: one cp.async load of the tile and one
// store of the factor.
#include "common.cuh"
#include "mma.cuh"

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

template <int SPLIT>
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
    const int g = lane >> 2, t = lane & 3;

    // load the lower triangle by block columns, 16-byte copies
    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        const int q = R / 4;                       // 16-byte pieces per column
        for (int e = tid; e < 32 * q; e += SM_THREADS) {
            const int cc = e / q, rr = (e - cc * q) * 4;
            cp_async_16(S + off + cc * ld + rr, T + (size_t)(32 * j + cc) * ldt + 32 * j + rr,
                        true);
        }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        float *P = S + off;                        // block column j, P[cc*ld + rr]
        // (a) diagonal block
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
                const float sd = ok ? sqrtf(d) : 1.f;
                const float rd = 1.f / sd;
                if (lane == c) myrd = rd;
                if (lane >= c) v[c] = lane == c ? sd : v[c] * rd;
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
        // (b) rows below the block: x D^T = a
        for (int rr = 32 + tid; rr < R; rr += SM_THREADS) {
            float x[32];
#pragma unroll
            for (int c = 0; c < 32; c++) x[c] = P[c * ld + rr];
            // column-oriented substitution: x_c final, then its multiple of
            // column c of the block leaves the later entries
#pragma unroll
            for (int c = 0; c < 32; c++) {
                x[c] *= rdiag[c];
#pragma unroll
                for (int c2 = c + 1; c2 < 32; c2++) x[c2] -= x[c] * P[c * ld + c2];
            }
#pragma unroll
            for (int c = 0; c < 32; c++) P[c * ld + rr] = x[c];
        }
        __syncthreads();
        // (c) trailing lower triangle: block columns j+1 .. nbc-1
        const int m = nbc - j - 1;
        const int npairs = m * (m + 1) / 2;
        for (int p = warp; p < npairs; p += SM_THREADS / 32) {
            int bj = 0, q = p;
            while (q >= m - bj) { q -= m - bj; bj++; }
            const int bi = bj + q;
            const int jc = j + 1 + bj;                       // block column of C
            float *C = S + col_off(nk, jc) + 32 * (bi - bj);  // C(i, c) = C[c*ldc + i]
            const int ldc = col_ld(nk, jc);
            const float *Xa = P + 32 * (1 + bi);             // rows of C
            const float *Xb = P + 32 * (1 + bj);             // columns of C
            float acc[2][4][4];
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 4; b++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;
#pragma unroll
            for (int k8 = 0; k8 < 32; k8 += 8) {
                float bf[4][2];
#pragma unroll
                for (int ni = 0; ni < 4; ni++) {
                    bf[ni][0] = Xb[(k8 + t) * ld + ni * 8 + g];
                    bf[ni][1] = Xb[(k8 + t + 4) * ld + ni * 8 + g];
                }
#pragma unroll
                for (int mi = 0; mi < 2; mi++) {
                    float af[4];
                    af[0] = Xa[(k8 + t) * ld + mi * 16 + g];
                    af[1] = Xa[(k8 + t) * ld + mi * 16 + g + 8];
                    af[2] = Xa[(k8 + t + 4) * ld + mi * 16 + g];
                    af[3] = Xa[(k8 + t + 4) * ld + mi * 16 + g + 8];
#pragma unroll
                    for (int ni = 0; ni < 4; ni++) mma8<SPLIT>(acc[mi][ni], af, bf[ni]);
                }
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const int r = mi * 16 + g + 8 * h, c = ni * 8 + 2 * t + e;
                            if (bi != bj || r >= c) C[c * ldc + r] -= acc[mi][ni][2 * h + e];
                        }
        }
        __syncthreads();
    }
    // store the factor (lower triangle)
    for (int j = 0; j < nbc; j++) {
        const int R = nk - 32 * j, ld = col_ld(nk, j), off = col_off(nk, j);
        for (int e = tid; e < 32 * R; e += SM_THREADS) {
            const int cc = e / R, rr = e - cc * R;
            if (rr >= cc) T[(size_t)(32 * j + cc) * ldt + 32 * j + rr] = S[off + cc * ld + rr];
        }
    }
}

template <int SPLIT>
void launch(cudaStream_t s, plasma_devstat_t *st, int call, const plasma_desc_t &A, int k,
            int iinfo, int bytes)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_potrf_diag_smem<SPLIT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem_floats(SM_NBMAX) * 4);
    }
    k_potrf_diag_smem<SPLIT><<<1, SM_THREADS, bytes, s>>>(A, k, iinfo, st, call);
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
    const int bytes = smem_floats(nk) * 4;
    if (split == 1) launch<1>(s, st, call, A, k, iinfo, bytes);
    else launch<3>(s, st, call, A, k, iinfo, bytes);
    return 1;
}
