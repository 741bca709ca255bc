// common.cuh -- device-side helpers shared by the tile kernels.
//
// Tiles are addressed through the descriptor arithmetic of
// plasma_descriptor.h (compiled for the device here).  Upper-triangular
// storage is handled by viewing every stored upper tile (n,m), n <= m, as the
// transpose of a logical lower tile (m,n): the kernels are written once for
// the lower algorithm of the reference (compute/pzpotrf.c:37-80) and the
// upper one (:84-126) is the same computation on transposed tiles.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../internal.h"

extern "C" long long plasma_launch_count_g;

#define PLASMA_COUNT_LAUNCH() (plasma_note_cuda_error(), ++plasma_launch_count_g)

// True the first time it is called with this flag word for the current
// device (bit d for device d).  Kernel attributes such as the dynamic shared
// memory limit belong to one device's context, so each is set once per device.
inline bool plasma_first_on_device(unsigned long long *mask)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (*mask & bit) return false;
    *mask |= bit;
    return true;
}

// A logical lower-storage view of one tile: element (i,j) of the logical tile
// is p[j*ld + i], or p[i*ld + j] when the stored tile is its transpose.
template <typename T>
struct TileView {
    T *p;
    int ld;
    int rows;   // logical rows
    int cols;   // logical cols
    bool trans;
    __device__ __forceinline__ T &at(int i, int j) const {
        return trans ? p[(size_t)i * ld + j] : p[(size_t)j * ld + i];
    }
};

// Logical lower tile (m,n), m >= n, of a triangular or general descriptor
// with storage `uplo` (PlasmaLower or PlasmaUpper).
template <typename T>
__device__ __forceinline__ TileView<T> tile_view(const plasma_desc_t &A,
                                                 int uplo, int m, int n)
{
    TileView<T> v;
    if (uplo == PlasmaUpper) {
        v.p = (T *)plasma_tile_addr(A, n, m);
        v.ld = plasma_tile_mmain(A, n);
        v.trans = true;
    } else {
        v.p = (T *)plasma_tile_addr(A, m, n);
        v.ld = plasma_tile_mmain(A, m);
        v.trans = false;
    }
    v.rows = plasma_tile_mview(A, m);
    v.cols = plasma_tile_mview(A, n);
    return v;
}

// Reads the status word; kernels return early once a failure was recorded,
// mirroring the "if (sequence->status == PlasmaSuccess)" test at the top of
// every reference task (core_blas/core_zpotrf.c:74).
__device__ __forceinline__ bool plasma_failed(const plasma_devstat_t *st)
{
    return *(volatile const int *)&st->status != 0;
}

// Records the first failure; later failures of the same sequence are ignored.
__device__ __forceinline__ void plasma_fail(plasma_devstat_t *st, int code,
                                            int call)
{
    if (atomicCAS(&st->status, 0, code) == 0)
        atomicExch(&st->call, call);
}

// ---------------------------------------------------------------------------
// cp.async (global -> shared, L1 bypass where possible) with zero fill
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async_8(void *sdst, const void *gsrc,
                                           bool valid)
{
    int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::
                 "r"(smem_u32(sdst)), "l"(gsrc), "r"(n));
}

__device__ __forceinline__ void cp_async_4(void *sdst, const void *gsrc,
                                           bool valid)
{
    int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::
                 "r"(smem_u32(sdst)), "l"(gsrc), "r"(n));
}

__device__ __forceinline__ void cp_async_16(void *sdst, const void *gsrc,
                                            bool valid)
{
    int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::
                 "r"(smem_u32(sdst)), "l"(gsrc), "r"(n));
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::);
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------------------
// FP64 tensor-core MMA (DMMA): D(16x8) += A(16x8) * B(8x8), FP64 throughout.
// Fragment ownership (lane = 4*g + t):
//   a0 (g, t)  a1 (g+8, t)  a2 (g, t+4)  a3 (g+8, t+4)
//   b0 (k=t, n=g)  b1 (k=t+4, n=g)
//   c0 (g, 2t) c1 (g, 2t+1) c2 (g+8, 2t) c3 (g+8, 2t+1)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4],
                                            const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

static inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
