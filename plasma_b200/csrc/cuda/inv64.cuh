// inv64.cuh -- the inverse of a 64 x 64 lower-triangular matrix in FP64, by
// one CTA of 256 threads in shared memory: the eight 8 x 8 diagonal blocks
// by substitution (a thread per column, in registers), then
// [A 0; B C]^-1 = [A^-1 0; -C^-1 B A^-1  C^-1] at sizes 16, 32 and 64, the
// products of the last two on DMMA.  Used for the diagonal blocks of the
// tensor-core panel solve (trsm_tc.cu) and of the LU (getrf.cu).
#pragma once
#include "common.cuh"

namespace {

// One warp: the 16 x 8 block C (+)= A (16 x K) B (K x 8) on DMMA, A and B
// row-major in shared memory (fragment layout of dmma_16x8x8).
__device__ __forceinline__ void warp_tile_f64(double (&c)[4], const double *A, int lda,
                                              const double *B, int ldb, int K)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int k0 = 0; k0 < K; k0 += 8) {
        const double af[4] = {A[g * lda + k0 + t], A[(g + 8) * lda + k0 + t],
                              A[g * lda + k0 + t + 4], A[(g + 8) * lda + k0 + t + 4]};
        const double bf[2] = {B[(k0 + t) * ldb + g], B[(k0 + t + 4) * ldb + g]};
        dmma_16x8x8(c, af, bf);
    }
}

// Ls: the matrix (lower part and diagonal; zero above), Iv: zero on entry,
// the inverse on exit (zero above the diagonal), Tm: scratch.  Called by
// all 256 threads of the CTA after the writes of Ls and Iv are visible
// (__syncthreads); returns after a __syncthreads.
__device__ __forceinline__ void inv_lower64(double (*Ls)[65], double (*Iv)[65],
                                            double (*Tm)[33], bool unit)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    double *rdiag = &Tm[48][0];                // 1 / L_ii (Tm rows 48 .. 63 are unused
                                               // until then)
    if (tid < 64) rdiag[tid] = unit ? 1.0 : 1.0 / Ls[tid][tid];
    __syncthreads();
    // the eight 8 x 8 diagonal blocks: a thread per column, in registers
    if (tid < 64) {
        const int o = tid & ~7, cc = tid & 7;
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            double s = i == cc ? 1.0 : 0.0;
#pragma unroll
            for (int q = 0; q < i; q++) s -= Ls[o + i][o + q] * x[q];
            x[i] = i >= cc ? s * rdiag[o + i] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 8; i++) Iv[o + i][o + cc] = x[i];
    }
    __syncthreads();
    // pairs [A 0; B C] of h x h blocks: the lower-left block of the inverse,
    // -C^-1 (B A^-1).  Iv is zero above its diagonal, so the products may
    // run over whole rows of the triangular factors.
    {   // h = 8: four pairs, a thread per entry
        const int p = tid / 64, i = (tid % 64) / 8, c = tid % 8, o = 16 * p;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; q++) s += Ls[o + 8 + i][o + q] * Iv[o + q][o + c];
        Tm[o + i][c] = s;
        __syncthreads();
        s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; q++) s += Iv[o + 8 + i][o + 8 + q] * Tm[o + q][c];
        Iv[o + 8 + i][o + c] = -s;
        __syncthreads();
    }
    {   // h = 16: two pairs, warps 0-3 each a 16 x 8 block of one pair
        const int p = warp >> 1, nt = warp & 1, o = 32 * p;
        if (warp < 4) {
            double c[4] = {0.0, 0.0, 0.0, 0.0};
            warp_tile_f64(c, &Ls[o + 16][o], 65, &Iv[o][o + 8 * nt], 65, 16);
#pragma unroll
            for (int e = 0; e < 4; e++) Tm[o + g + 8 * (e >> 1)][8 * nt + 2 * t + (e & 1)] = c[e];
        }
        __syncthreads();
        if (warp < 4) {
            double c[4] = {0.0, 0.0, 0.0, 0.0};
            warp_tile_f64(c, &Iv[o + 16][o + 16], 65, &Tm[o][8 * nt], 33, 16);
#pragma unroll
            for (int e = 0; e < 4; e++)
                Iv[o + 16 + g + 8 * (e >> 1)][o + 8 * nt + 2 * t + (e & 1)] = -c[e];
        }
        __syncthreads();
    }
    {   // h = 32: one pair, warp w the 16 x 8 block (w / 4, w mod 4)
        const int mt = warp >> 2, nt = warp & 3;
        double c[4] = {0.0, 0.0, 0.0, 0.0};
        warp_tile_f64(c, &Ls[32 + 16 * mt][0], 65, &Iv[0][8 * nt], 65, 32);
#pragma unroll
        for (int e = 0; e < 4; e++) Tm[16 * mt + g + 8 * (e >> 1)][8 * nt + 2 * t + (e & 1)] = c[e];
        __syncthreads();
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        warp_tile_f64(d, &Iv[32 + 16 * mt][32], 65, &Tm[0][8 * nt], 33, 32);
#pragma unroll
        for (int e = 0; e < 4; e++)
            Iv[32 + 16 * mt + g + 8 * (e >> 1)][8 * nt + 2 * t + (e & 1)] = -d[e];
        __syncthreads();
    }
}

}  // namespace
