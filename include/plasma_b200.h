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

/* Number of device (cudaMalloc) and page-locked host (cudaMallocHost)
 * allocations this library has made since the process started. */
long long plasma_device_allocations(void);

/* Tile size the PlasmaTuning table holds for the size bucket of n
 * (dtyp = PlasmaRealDouble or PlasmaRealFloat), and its update by a measured
 * autotuner. */
int plasma_tuning_get_potrf_nb(int dtyp, int n);
int plasma_tuning_set_potrf_nb(int dtyp, int n, int nb);
/* Measured autotuning of the tables above (no reference counterpart: the
 * reference reads nb from a Lua script).  plasma_autotune_potrf times the
 * tile factorization of a synthetic SPD matrix of order n for nb in
 * {128, 256, 384, 512}, stores the fastest for n's size bucket and returns
 * it (its time in *best_ms when not NULL).  plasma_autotune_batched times
 * batches of `count` matrices of each bucket's largest order with block
 * widths 16 and 32 and stores the faster per bucket.  Negative returns:
 * argument position or PlasmaError*. */
int plasma_autotune_potrf(plasma_enum_t dtyp, int n, double *best_ms);
int plasma_autotune_batched(plasma_enum_t dtyp, int count);
/* Block width (16 or 32) of the batched kernels for matrices of order n. */
int plasma_tuning_get_batched_nb(int dtyp, int n);
int plasma_tuning_set_batched_nb(int dtyp, int n, int nb);

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
 * capture.  All calls share the one array and a per-device epoch counter
 * (host memory): calls that overlap (other streams, other host threads)
 * race on both, and the array keeps the last call's contents (each sweep
 * clears its own ticket and abort words; the flags are matched against the
 * call's epoch, not against zero).
 */
#define PLASMA_NOALLOC_MAX_N 8192
void plasma_omp_dpotrs_noalloc(plasma_enum_t uplo, plasma_desc_t A,
                               plasma_desc_t B, plasma_sequence_t *sequence,
                               plasma_request_t *request);

/*
 * Reverse mode of the Cholesky factor and solve.  No reference counterpart
 * (PLASMA computes no derivatives).  A = L L^T (uplo = PlasmaLower) or
 * A = U^T U (PlasmaUpper, L = U^T).
 *
 * plasma_?potrf_adjoint: on entry the uplo triangle of Lbar holds the
 * cotangent of the factor; on exit Lbar holds the full symmetric cotangent of
 * A, sym(L^-T Phi(L^T Lbar) L^-1) with Phi the lower triangle and half the
 * diagonal (both triangles written).  Returns -1/-2/-4/-6 for an illegal
 * uplo/n/ldl/ldlbar.
 *
 * plasma_?potrs_adjoint: X = A^-1 B was computed with the factor in L.  On
 * entry Xbar is the cotangent of X, on exit the cotangent of B (A^-1 Xbar);
 * the uplo triangle of Lbar is decreased by the factor cotangent of the
 * solve, tril((Bbar X^T + X Bbar^T) L) (its transpose for upper storage), so
 * that the cotangents of several uses of L accumulate in Lbar before one
 * plasma_?potrf_adjoint.  Returns -1/-2/-3/-5/-7/-9/-11 for an illegal
 * uplo/n/nrhs/ldl/ldx/ldxbar/ldlbar.
 *
 * Pointers may be host or device memory.  The omp forms take general
 * descriptors (Lbar general for potrf_adjoint) and report through sequence.
 */
int plasma_dpotrf_adjoint(plasma_enum_t uplo, int n, const double *pL, int ldl,
                          double *pLbar, int ldlbar);
int plasma_spotrf_adjoint(plasma_enum_t uplo, int n, const float *pL, int ldl,
                          float *pLbar, int ldlbar);
int plasma_dpotrs_adjoint(plasma_enum_t uplo, int n, int nrhs, const double *pL, int ldl,
                          const double *pX, int ldx, double *pXbar, int ldxbar,
                          double *pLbar, int ldlbar);
int plasma_spotrs_adjoint(plasma_enum_t uplo, int n, int nrhs, const float *pL, int ldl,
                          const float *pX, int ldx, float *pXbar, int ldxbar,
                          float *pLbar, int ldlbar);
void plasma_omp_dpotrf_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_omp_spotrf_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_omp_dpotrs_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t X,
                               plasma_desc_t Xbar, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_omp_spotrs_adjoint(plasma_enum_t uplo, plasma_desc_t L, plasma_desc_t X,
                               plasma_desc_t Xbar, plasma_desc_t Lbar,
                               plasma_sequence_t *sequence, plasma_request_t *request);

/*
 * Batched SPD systems of uneven order (0 <= n_i <= 512).  No reference
 * counterpart (PLASMA factors one matrix at a time).  A plan fixes the
 * orders: matrix i is column-major n_i x n_i (ld n_i) at element offset
 * off_a[i] of one device array, its vector (one right-hand side) at off_b[i]
 * of another (plasma_batch_offsets; plasma_batch_matrix_elems /
 * plasma_batch_vector_elems give the array lengths).  Each operation is one
 * persistent kernel launch on the context stream (device pointers, returns
 * at once); the plan orders the matrices largest first and takes the block
 * width of each size bucket from the tuning table.  With
 * plasma_batch_set_graph(plan, 1) the launch is captured once into a CUDA
 * graph held by the plan and replayed by later calls with the same
 * pointers.
 *   posv    : A <- L (lower triangle), B <- A^-1 B, info[i] as LAPACK dpotrf
 *             (the solve is skipped for a matrix with info != 0)
 *   potrf   : A <- L, info
 *   potrs   : B <- A^-1 B with the factor in L
 *   potrf_adjoint : Lbar (cotangent of L in the lower triangle) <- the
 *             symmetric cotangent of A, both triangles
 *   potrs_adjoint : Xbar <- A^-1 Xbar, lower triangle of Lbar -=
 *             tril((Bbar X^T + X Bbar^T) L)
 * Returns 0, PlasmaErrorNotInitialized, or a negative argument position.
 */
typedef struct plasma_batch_s plasma_batch_t;
int plasma_batch_create(plasma_enum_t precision, int batch, const int *n,
                        plasma_batch_t **plan);
void plasma_batch_destroy(plasma_batch_t *plan);
long long plasma_batch_matrix_elems(const plasma_batch_t *plan);
long long plasma_batch_vector_elems(const plasma_batch_t *plan);
int plasma_batch_offsets(const plasma_batch_t *plan, long long *off_a, long long *off_b);
int plasma_batch_set_graph(plasma_batch_t *plan, int on);
int plasma_dposv_batched(plasma_batch_t *plan, double *A, double *B, int *info);
int plasma_sposv_batched(plasma_batch_t *plan, float *A, float *B, int *info);
int plasma_dpotrf_batched(plasma_batch_t *plan, double *A, int *info);
int plasma_spotrf_batched(plasma_batch_t *plan, float *A, int *info);
int plasma_dpotrs_batched(plasma_batch_t *plan, const double *L, double *B);
int plasma_spotrs_batched(plasma_batch_t *plan, const float *L, float *B);
int plasma_dpotrf_adjoint_batched(plasma_batch_t *plan, const double *L, double *Lbar);
int plasma_spotrf_adjoint_batched(plasma_batch_t *plan, const float *L, float *Lbar);
int plasma_dpotrs_adjoint_batched(plasma_batch_t *plan, const double *L, const double *X,
                                  double *Xbar, double *Lbar);
int plasma_spotrs_adjoint_batched(plasma_batch_t *plan, const float *L, const float *X,
                                  float *Xbar, float *Lbar);

/* Human-readable name of a return code. */
const char *plasma_strerror(int code);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_B200_H */
