// mma.cuh -- m16n8k8 tensor-core steps shared by the panel, adjoint and
// batched kernels: DMMA for FP64, TF32 mma.sync for FP32, once or as the
// FP32-accurate three-product split.
#pragma once
#include "common.cuh"

namespace {

// m16n8k8 tensor-core step with the FP64 fragment layout of dmma_16x8x8.
// double: DMMA.  float: TF32 mma.sync, either once (SPLIT = 1) or as the
// three-term split a = a_hi + a_lo (SPLIT = 3: a_hi b_hi + a_hi b_lo +
// a_lo b_hi), which keeps FP32-level accuracy.
__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void tf32_mma(float (&c)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int SPLIT>
__device__ __forceinline__ void mma8(double (&c)[4], const double (&a)[4],
                                     const double (&b)[2])
{
    dmma_16x8x8(c, a, b);
}

template <int SPLIT>
__device__ __forceinline__ void mma8(float (&c)[4], const float (&a)[4],
                                     const float (&b)[2])
{
    uint32_t ah[4], bh[2];
#pragma unroll
    for (int i = 0; i < 4; i++) ah[i] = to_tf32(a[i]);
#pragma unroll
    for (int i = 0; i < 2; i++) bh[i] = to_tf32(b[i]);
    if (SPLIT == 3) {
        uint32_t al[4], bl[2];
#pragma unroll
        for (int i = 0; i < 4; i++) al[i] = to_tf32(a[i] - __uint_as_float(ah[i]));
#pragma unroll
        for (int i = 0; i < 2; i++) bl[i] = to_tf32(b[i] - __uint_as_float(bh[i]));
        tf32_mma(c, al, bh);
        tf32_mma(c, ah, bl);
    }
    tf32_mma(c, ah, bh);
}

// Row strides (elements) that make the fragment loads conflict-free:
// 4 mod 16 for 8-byte elements, 8 mod 32 for 4-byte elements.
template <typename T> struct Pad { static constexpr int v = 4; };
template <> struct Pad<float> { static constexpr int v = 8; };

template <typename T>
__device__ __forceinline__ void cp_async_el(T *dst, const T *src, bool v)
{
    if (sizeof(T) == 8) cp_async_8(dst, src, v);
    else cp_async_4(dst, src, v);
}

}  // namespace
