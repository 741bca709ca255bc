/*
 * tuning.c -- tile-size selection behind the PlasmaTuning switch.
 *
 * The reference asks a Lua script for nb (plasma_tune_potrf / plasma_tune_trsm,
 * control/tuning.c:367-374,427-434; potrf_nb returns 256 in
 * tuning/default.lua:125-127) and, like here, writes the answer into the
 * context's nb.  Without a script nb stays at the plasma_set value.
 *
 * The GPU build keeps small tables of tile sizes per (precision, size
 * bucket): nb of the tile factorization and the block width of the batched
 * kernels.  They start from built-in defaults and are refreshed at run time
 * by the measured autotuner (cuda/autotune.cu: plasma_autotune_potrf,
 * plasma_autotune_batched).
 */
#include "../internal.h"

#include <stdlib.h>

#define NBUCKETS 8

/* bucket b covers n < 1024 << b (the last bucket is open-ended) */
static int bucket_of(int n)
{
    int b = 0;
    while (b < NBUCKETS - 1 && n >= (1024 << b))
        b++;
    return b;
}

/* [0] FP64, [1] FP32; 0 = no entry (keep plasma->nb) */
static int potrf_table[2][NBUCKETS] = {
    /* <1k  <2k  <4k  <8k  <16k <32k <64k  rest */
    {  128, 128, 256, 256, 256, 256, 256,  256 },
    {  128, 256, 256, 256, 256, 256, 256,  256 },
};

static int prec_index(plasma_enum_t dtyp)
{
    return dtyp == PlasmaRealDouble || dtyp == PlasmaComplexDouble ? 0 : 1;
}

void plasma_tune_potrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n)
{
    const char *env = getenv("PLASMA_TUNING_DISABLE");
    if (env && env[0] == '1')
        return;
    int nb = potrf_table[prec_index(dtyp)][bucket_of(n)];
    if (nb > 0)
        plasma->nb = nb;
}

/* Band factorization and solves (the reference's plasma_tune_pbtrf,
 * control/tuning.c:347-354, pbtrf_nb = 256 in tuning/default.lua:120-122).
 * Here the band walk is a chain of n/nb dependent tile steps, and what a
 * step costs grows with nb faster than the step count falls: measured on
 * B200 at n = 32768, kd in {256, 1024, 4096}, nb = 128 is the fastest in
 * FP64 at every kd and in FP32 up to kd = 1024; FP32 at kd = 4096 prefers
 * 256 (its trailing windows are large enough to keep the SMs busy). */
void plasma_tune_pbtrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n, int kd)
{
    (void)n;
    const char *env = getenv("PLASMA_TUNING_DISABLE");
    if (env && env[0] == '1')
        return;
    plasma->nb = (dtyp == PlasmaRealFloat && kd >= 2048) ? 256 : 128;
}

void plasma_tune_trsm(plasma_context_t *plasma, plasma_enum_t dtyp, int m,
                      int n)
{
    (void)n;
    plasma_tune_potrf(plasma, dtyp, m);
}

/* Stores nb for the size bucket of n (GPU-build extension, used by the
 * measured autotuner). */
int plasma_tuning_set_potrf_nb(int dtyp, int n, int nb)
{
    if (nb <= 0 || nb > 1024)
        return PlasmaErrorIllegalValue;
    potrf_table[prec_index(dtyp)][bucket_of(n)] = nb;
    return PlasmaSuccess;
}

int plasma_tuning_get_potrf_nb(int dtyp, int n)
{
    return potrf_table[prec_index(dtyp)][bucket_of(n)];
}

/* Block width of the batched kernels (16 or 32) per size bucket of the
 * matrix order: buckets n <= 32, 64, 128, 256, 512.  [0] FP64, [1] FP32. */
#define NBBUCKETS 5
static int batched_table[2][NBBUCKETS] = {
    /* <=32 <=64 <=128 <=256 <=512 */
    {  32,  16,  32,   32,   32 },
    {  32,  16,  32,   32,   32 },
};

static int batched_bucket(int n)
{
    int b = 0;
    while (b < NBBUCKETS - 1 && n > (32 << b))
        b++;
    return b;
}

int plasma_tuning_get_batched_nb(int dtyp, int n)
{
    return batched_table[prec_index(dtyp)][batched_bucket(n)];
}

int plasma_tuning_set_batched_nb(int dtyp, int n, int nb)
{
    if (nb != 16 && nb != 32)
        return PlasmaErrorIllegalValue;
    batched_table[prec_index(dtyp)][batched_bucket(n)] = nb;
    return PlasmaSuccess;
}
