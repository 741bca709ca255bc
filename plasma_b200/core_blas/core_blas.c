/*
 * core_blas.c -- libplasma_core_blas.so: the reference's CPU tile kernels
 * (plasma_core_{d,s}{potrf,trsm,syrk,gemm,symm,lacpy,geadd,lange,lansy},
 * plasma_core_dlag2s, plasma_core_slag2d, plasma_core_omp_{d,s}amax;
 * include/plasma_core_blas_z.h, plasma_core_blas_zc.h of the reference) with
 * their host-memory semantics, so that code written against the reference's
 * kernel-substitution interface links and runs.  A compatibility library:
 * the GPU library libplasma_b200.so neither links nor calls it.
 */
#include <float.h>
#include <math.h>
#include <stddef.h>

#include "plasma_core_blas.h"

#define REAL double
#define X(name) plasma_core_d##name
#define OMPX(name) plasma_core_omp_d##name
#include "core_blas_impl.h"
#undef REAL
#undef X
#undef OMPX

#define REAL float
#define X(name) plasma_core_s##name
#define OMPX(name) plasma_core_omp_s##name
#include "core_blas_impl.h"
#undef REAL
#undef X
#undef OMPX

/* LAPACK dlag2s (core_zlag2c.c:48-60): As <- (float) A; returns 1 at the
 * first entry outside the FP32 range (the conversion stops there). */
int plasma_core_dlag2s(int m, int n, const double *A, int lda, float *As, int ldas)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            const double v = A[(size_t)j * lda + i];
            if (v < -FLT_MAX || v > FLT_MAX)
                return 1;
            As[(size_t)j * ldas + i] = (float)v;
        }
    return 0;
}

/* LAPACK slag2d (core_clag2z.c:48-68): A <- (double) As */
void plasma_core_slag2d(int m, int n, const float *As, int ldas, double *A, int lda)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++)
            A[(size_t)j * lda + i] = (double)As[(size_t)j * ldas + i];
}
