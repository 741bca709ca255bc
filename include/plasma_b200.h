/*
 * plasma_b200.h -- additions of the B200 build that have no counterpart in
 * the reference API.  Plain C types only (pointers, sizes, ints), so that the
 * header can be bound from C, Fortran (ISO_C_BINDING) or Python ctypes.
 */
#ifndef PLASMA_B200_H
#define PLASMA_B200_H

#include "plasma_types.h"
#include "plasma_descriptor.h"
#include "plasma_async.h"

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Outcome of a mixed-precision solve, filled by plasma_dsposv_ex(). */
typedef struct {
    int    factor_mode;     /* PlasmaFactor* actually used for the factor    */
    int    refinement;      /* PlasmaRefine* actually used                   */
    int    ir_iterations;   /* outer refinement iterations                   */
    int    gmres_iterations;/* total inner GMRES iterations (GMRES-IR only)  */
    int    fallback_fp64;   /* 1 if the FP64 factorisation was used          */
    int    attempts;        /* number of factor precisions tried            */
    double backward_error;  /* max_j ||b_j - A x_j||_inf /
                               (||A||_inf ||x_j||_inf)                       */
    double anorm;           /* ||A||_inf                                     */
    double factor_ms;       /* device time of the low-precision factor       */
    double refine_ms;       /* device time of the refinement                 */
} plasma_dsposv_info_t;

/*
 * plasma_dsposv with a report and the extended modes (TF32 / BF16 factors,
 * GMRES-IR, automatic escalation BF16 -> TF32 -> FP32 -> FP64).  Same return
 * values and *iter convention as plasma_dsposv.  info may be NULL.
 */
int plasma_dsposv_ex(plasma_enum_t uplo, int n, int nrhs,
                     double *pA, int lda, double *pB, int ldb,
                     double *pX, int ldx, int *iter,
                     plasma_dsposv_info_t *info);

/* CUDA stream (a cudaStream_t passed as void*) the context enqueues on;
 * NULL restores the context's own stream. */
int plasma_set_stream(void *stream);
void *plasma_get_stream(void);

/* Number of kernels this library has launched since plasma_init(). */
long long plasma_kernel_launches(void);

/* Tile size the PlasmaTuning table holds for the size bucket of n
 * (dtyp = PlasmaRealDouble or PlasmaRealFloat), and its update by a measured
 * autotuner. */
int plasma_tuning_get_potrf_nb(int dtyp, int n);
int plasma_tuning_set_potrf_nb(int dtyp, int n, int nb);

/* Kernel classes of the opt-in profiler. */
enum {
    PLASMA_KCLASS_POTRF  = 0,   /* diagonal-tile Cholesky                   */
    PLASMA_KCLASS_TRSM   = 1,   /* panel solve                              */
    PLASMA_KCLASS_UPDATE = 2,   /* trailing SYRK/GEMM update                */
    PLASMA_KCLASS_SOLVE  = 3,   /* triangular solve sweeps (potrs)          */
    PLASMA_KCLASS_AUX    = 4,   /* norms, residual, conversions, layout     */
    PLASMA_KCLASS_COUNT  = 5
};

/* Profiling: when enabled, every tile-step launch is bracketed by CUDA events
 * on its own stream; query returns, per class, the launches, the summed
 * device milliseconds and the algorithmic flops and bytes of those launches.
 * Enabling (or re-enabling) resets the counters. */
void plasma_profile_enable(int on);
int plasma_profile_query(int kclass, long long *launches, double *ms,
                         double *flops, double *bytes);

/*
 * No reference counterpart.  plasma_omp_dpotrs for one right-hand side
 * (A: FP64 Cholesky factor in square tiles, nb a multiple of 64; B: n x 1)
 * for callers that cannot allocate device memory while they solve (device
 * memory owned by another allocator, or a latency-bound loop where
 * cudaMalloc/cudaFree would synchronise the device).  It takes no device
 * memory from the library: its scratch (the inverses
 * of the 64 x 64 diagonal blocks and the sweep ready flags) is a file-scope
 * device array of 4 MiB + 4 KiB, so n <= PLASMA_NOALLOC_MAX_N.  Larger n
 * fails the request with PlasmaErrorIllegalValue, other shapes with
 * PlasmaErrorNotSupported.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the one array: calls that overlap (other
 * streams, other host threads) race, and the array keeps the last call's
 * contents (each sweep clears its own ticket and abort words; the flags are
 * matched against a per-call epoch, not against zero).
 */
#define PLASMA_NOALLOC_MAX_N 8192
void plasma_omp_dpotrs_noalloc(plasma_enum_t uplo, plasma_desc_t A,
                               plasma_desc_t B, plasma_sequence_t *sequence,
                               plasma_request_t *request);

/* Human-readable name of a return code. */
const char *plasma_strerror(int code);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_B200_H */
