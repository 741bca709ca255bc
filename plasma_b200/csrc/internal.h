/*
 * internal.h -- declarations shared by the C host layer (control/, compute/)
 * and the CUDA launch layer (cuda/).  Nothing here is part of the public ABI.
 *
 * Execution model.  The reference opens "omp parallel / omp master" and turns
 * every tile operation into an OpenMP task whose depend() clauses form the DAG
 * (compute/pzpotrf.c:37-80, core_blas/core_zgemm.c:125-127).  Here the host
 * walks the same loops but launches one CUDA kernel per *tile step*
 * (all TRSMs of a panel, all SYRK/GEMM updates of a step) and orders them with
 * CUDA streams and events.  The cooperative cancellation of the reference
 * (every task tests sequence->status, core_blas/core_zpotrf.c:74) becomes a
 * device status word that every kernel reads first and that the failing kernel
 * writes.
 */
#ifndef PLASMA_B200_INTERNAL_H
#define PLASMA_B200_INTERNAL_H

#include "plasma.h"
#include "plasma_b200.h"

#include <cuda_runtime_api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Device status word shared by all kernels of a context. */
typedef struct {
    int status;   /* 0 = running fine; > 0 = LAPACK-style info; < 0 = error */
    int call;     /* id of the plasma_omp_* call whose kernel failed       */
    int spare[2];
} plasma_devstat_t;

#define PLASMA_MAX_PENDING_CALLS 4096
/* aux[0]: critical path, aux[1]: bulk updates, aux[2]: uploads,
 * aux[3 ..]: one update stream per group of arriving tile columns */
#define PLASMA_NUM_STREAMS 16
#define PLASMA_STREAM_COPY 2
#define PLASMA_GROUP_STREAMS (PLASMA_NUM_STREAMS - 3)
#define PLASMA_MAX_GROUPS 32     /* column groups of an arriving matrix */
#define PLASMA_STAGE_STREAMS 4   /* copies of pageable host blocks       */
#define PLASMA_SCRATCH_SLOTS 9

/* scratch slots */
enum {
    PLASMA_SLOT_STAGING = 0,   /* column-major copies of host operands       */
    PLASMA_SLOT_WORK    = 1,   /* inverses of diagonal tiles, panels          */
    PLASMA_SLOT_SMALL   = 2,   /* norms and other vectors                     */
    PLASMA_SLOT_MIXED   = 3,   /* low-precision operand copies (dsposv)       */
    PLASMA_SLOT_REFINE  = 4,   /* refinement vectors and Krylov basis         */
    PLASMA_SLOT_SYMV    = 5,   /* per-tile partial products of the residual   */
    PLASMA_SLOT_ADJOINT = 6,   /* n x n work matrices of the adjoints         */
    PLASMA_SLOT_DESC_A  = 7,   /* dsposv's FP64 tile copy of A (kept)         */
    PLASMA_SLOT_DESC_AS = 8    /* dsposv's FP32 tile copy of A (kept)         */
};

typedef struct {
    int tuning;
    int nb;
    int ib;
    plasma_enum_t inplace_outplace;
    int max_threads;
    int max_panel_threads;
    plasma_enum_t householder_mode;

    /* GPU-build state */
    int device;
    int mixed_mode;      /* PlasmaFactor* */
    int refinement;      /* PlasmaRefine* */
    int lookahead;       /* >= 0 */
    int num_sms;
    cudaStream_t stream;                     /* the sequence stream         */
    cudaStream_t own_stream;                 /* created by plasma_init()    */
    cudaStream_t aux[PLASMA_NUM_STREAMS];    /* look-ahead / update streams */
    cudaStream_t stage[PLASMA_STAGE_STREAMS];/* pageable-host staging       */
    cudaEvent_t ev_stage[PLASMA_STAGE_STREAMS];
    cudaEvent_t ev_stage_in;
    unsigned stage_next;                     /* round robin over stage[]    */
    plasma_devstat_t *dstat;                 /* device status word          */
    plasma_devstat_t *dquiet;                /* a status word no kernel sets
                                                (work that must complete)  */
    plasma_devstat_t *hstat;                 /* pinned host mirror          */

    /* ids of plasma_omp_* calls since the last plasma_sequence_wait() */
    int next_call;
    plasma_request_t *pending[PLASMA_MAX_PENDING_CALLS];
    plasma_sequence_t *pending_seq[PLASMA_MAX_PENDING_CALLS];

    /* growable device scratch slots (never shrink until finalize) */
    void  *scratch[PLASMA_SCRATCH_SLOTS];
    size_t scratch_bytes[PLASMA_SCRATCH_SLOTS];
    void  *pinned;
    size_t pinned_bytes;
    cudaEvent_t ev[8];                        /* DAG edges (reused)        */
    cudaEvent_t ev_group[PLASMA_MAX_GROUPS]; /* arrival of column groups   */
    /* ready flags of the one-launch triangular sweeps */
    void  *sweep_sync;
    size_t sweep_sync_bytes;
    int    sweep_epoch;
} plasma_context_t;

plasma_context_t *plasma_context_self(void);

/* Opt-in profiling (control/profile.c): brackets one launch on stream s. */
int plasma_prof_begin(cudaStream_t s);
void plasma_prof_end(int slot, cudaStream_t s, int kclass, double flops,
                     double bytes);

/* CUDA errors that no return code reports (a kernel launch with a bad
 * configuration, e.g. more dynamic shared memory than its limit, only
 * reaches the host through cudaGetLastError): plasma_note_cuda_error()
 * keeps the first one (allocation failures excepted: their callers
 * report them), plasma_take_cuda_error() returns and clears it.  Called
 * before every launch (PLASMA_COUNT_LAUNCH), before and after every
 * allocation, and by plasma_sequence_wait, which fails the sequence with
 * PlasmaErrorInternal. */
void plasma_note_cuda_error(void);
int plasma_take_cuda_error(void);
/* device and pinned allocations made by the library (plasma_device_allocations) */
extern long long plasma_alloc_count_g;

/* Registers a plasma_omp_* call; returns the id its kernels report. */
int plasma_call_begin(plasma_context_t *plasma, plasma_sequence_t *sequence,
                      plasma_request_t *request);

/* Device scratch of at least `bytes` in one of the slots above.  The buffer
 * stays valid until the same slot is requested with a larger size; all users
 * are ordered on the context streams, and growth waits for them. */
void *plasma_scratch(plasma_context_t *plasma, int slot, size_t bytes);
void *plasma_pinned(plasma_context_t *plasma, size_t bytes);

/* Queries whether p is device memory of the context's device. */
int plasma_is_device_pointer(const void *p);
/* Host memory that is neither page-locked nor registered with CUDA. */
int plasma_is_pageable(const void *p);

/* Host <-> device copies of column-major blocks (cudaMemcpy2DAsync
 * arguments; width in bytes, height in columns) through page-locked
 * staging slots when the host side is pageable (control/staging.c). */
void plasma_stage_begin(plasma_context_t *plasma, cudaStream_t s);
void plasma_stage_copy(plasma_context_t *plasma, void *dst, size_t dpitch, const void *src,
                       size_t spitch, size_t width, size_t height, enum cudaMemcpyKind kind);
void plasma_stage_join(plasma_context_t *plasma, cudaStream_t s);
void plasma_copy_2d(plasma_context_t *plasma, cudaStream_t s, void *dst, size_t dpitch,
                    const void *src, size_t spitch, size_t width, size_t height,
                    enum cudaMemcpyKind kind, int pageable);

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ----------------------------------------------------------------------------
 * Tile-step kernels (cuda/ directory).  Every launcher takes the stream, the
 * device status word and -- for kernels that can fail -- the call id.
 * prec is PlasmaRealDouble or PlasmaRealFloat.
 * ------------------------------------------------------------------------- */

/* Column-major (ld) <-> tile layout of the view of A.  For uplo = Lower/Upper
 * only the tiles of that triangle are copied (reference compute/pztr2desc.c). */
void plasma_cuda_lapack_to_tile(cudaStream_t s, plasma_devstat_t *st,
                                plasma_desc_t A, plasma_enum_t uplo,
                                const void *pA, int lda);
void plasma_cuda_tile_to_lapack(cudaStream_t s, plasma_devstat_t *st,
                                plasma_desc_t A, plasma_enum_t uplo,
                                void *pA, int lda);
/* The upper triangle of the column-major pA <-> the lower tiles of B,
 * transposed (an upper-stored matrix factored through lower tiles). */
void plasma_cuda_lapack_to_tile_t(cudaStream_t s, plasma_devstat_t *st,
                                  plasma_desc_t B, const void *pA, int lda);
void plasma_cuda_tile_to_lapack_t(cudaStream_t s, plasma_devstat_t *st,
                                  plasma_desc_t B, void *pA, int lda);
/* LAPACK-layout <-> tile conversions of an upper-stored array through lower
 * tiles (compute/transfer.c) */
void plasma_omp_Xlapack2desc_t(const void *pA, int lda, plasma_desc_t A,
                               plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_omp_Xdesc2lapack_t(plasma_desc_t A, void *pA, int lda,
                               plasma_sequence_t *sequence, plasma_request_t *request);
/* LAPACK band storage (ldab >= kd+1) <-> band tile descriptor of lower or
 * upper storage (reference compute/pzpb2desc.c, pzdesc2pb.c). */
void plasma_cuda_band_to_tile(cudaStream_t s, plasma_devstat_t *st,
                              plasma_desc_t A, const void *pAB, int ldab);
void plasma_cuda_tile_to_band(cudaStream_t s, plasma_devstat_t *st,
                              plasma_desc_t A, void *pAB, int ldab);

/* All diagonal-tile inverses W_k = inv(L_kk) (lower logical view) into W
 * (A.mt tiles of A.mb x A.mb, column-major). */
void plasma_cuda_trtri_tiles(cudaStream_t s, plasma_devstat_t *st,
                             plasma_enum_t uplo, plasma_desc_t A, void *W);

/* op(L) X = B in place (trans = PlasmaNoTrans or PlasmaTrans); W as above,
 * computed first when have_w == 0. */
/* One update step of a many-rhs tile sweep on the tensor cores (FP64 DMMA,
 * FP32 three-product TF32); 0 when the tiling does not fit (cuda/update.cu). */
int plasma_cuda_sweep_update_mma(cudaStream_t s, plasma_devstat_t *st,
                                  plasma_enum_t uplo, int trans, plasma_desc_t L,
                                  plasma_desc_t B, int k, int mlo, int mhi);
void plasma_cuda_trsm_sweep(cudaStream_t s, plasma_devstat_t *st,
                            plasma_enum_t uplo, plasma_enum_t trans,
                            plasma_desc_t A, plasma_desc_t B,
                            void *W, int have_w);

/* Diagonal-tile Cholesky of tile (k,k) (uplo Lower or Upper), writing
 * info = iinfo + j on a non-positive pivot in column j (1-based).  If winv is
 * not NULL it also receives W = inv(L_kk) (lower, ld = nb) used by the
 * panel solve. */
void plasma_cuda_potrf_tile(cudaStream_t s, plasma_devstat_t *st, int call,
                            plasma_enum_t uplo, plasma_desc_t A, int k,
                            int iinfo, void *winv);

/* Panel solve of step k: A(m,k) <- A(m,k) * L_kk^{-T} for m = k+1..mt-1
 * (upper: A(k,m) <- U_kk^{-T} A(k,m)), given W = inv(L_kk). mlo..mhi-1 is the
 * tile range processed. */
/* Panel solve of step k on the tensor cores (FP32, lower, tiles of 128 or
 * 256); writes the update's rounded panel copies when the mode's operands
 * are TF32.  0: not eligible, 1: solved, 2: solved and copies written. */
int plasma_cuda_trsm_tc(cudaStream_t s, plasma_devstat_t *st, int mode, plasma_desc_t A,
                        int k, int mlo, int mhi, void *wimg, void *panel, int full);
size_t plasma_cuda_trsm_tc_bytes(int nb);
/* Block inverses for the one-launch sweeps with an LU factor (unit-lower L
 * forward, U backward); 0 when the sweep block is not 64 rows. */
int plasma_cuda_trtri_blocks_lu(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                                void *Wf, void *Wb);
void plasma_cuda_trsm_panel(cudaStream_t s, plasma_devstat_t *st,
                            plasma_enum_t uplo, plasma_desc_t A, int k,
                            int mlo, int mhi, const void *winv);

/* Trailing update of step k restricted to tile columns n in [nlo, nhi) and
 * rows m >= n:  A(m,n) -= A(m,k) A(n,k)^T (SYRK on the diagonal, GEMM below).
 */
void plasma_cuda_update(cudaStream_t s, plasma_devstat_t *st,
                        plasma_enum_t uplo, plasma_desc_t A, int k,
                        int nlo, int nhi, int num_sms);

/* dsposv helpers. */
/* Infinity norm of symmetric A (uplo triangle) into *dnorm (device); work
 * (plasma_cuda_symv_work bytes, or NULL for the slow row-per-thread kernel)
 * selects the one-pass tile kernel. */
int plasma_cuda_lansy_tiles(cudaStream_t s, plasma_devstat_t *st,
                            plasma_enum_t uplo, plasma_desc_t A, double *norm,
                            double *work);
void plasma_cuda_lansy_inf(cudaStream_t s, plasma_devstat_t *st,
                           plasma_enum_t uplo, plasma_desc_t A,
                           double *dnorm, double *work);
/* info = i + 1 for the first zero A(i,i) of a triangular factor (dtrtri). */
void plasma_cuda_diag_zero_info(cudaStream_t s, plasma_devstat_t *st, int call,
                                plasma_desc_t A);
/* A <- uplo triangle of B (same tiling; the other triangle of A kept). */
void plasma_cuda_copy_uplo(cudaStream_t s, plasma_devstat_t *st, plasma_enum_t uplo,
                           plasma_desc_t B, plasma_desc_t A);
/* Tile columns [n0, n1) of a host upload in flight: FP64 tiles of A (lower)
 * from the column-major device copy src (leading dimension ld) and their
 * FP32 conversion into As (dlag2s overflow test), in one pass that runs
 * whatever the device status says. */
void plasma_cuda_upload_cols(cudaStream_t s, plasma_devstat_t *st, int call,
                             plasma_desc_t A, plasma_desc_t As, const double *src,
                             int ld, int n0, int n1);
/* As (lower tiles) <- (float)A with A in upper storage (transposed tiles). */
void plasma_cuda_lag2s_upper_to_lower(cudaStream_t s, plasma_devstat_t *st, int call,
                                      plasma_desc_t A, plasma_desc_t As);
/* As <- (float)A tile by tile; sets status 1 on overflow (dlag2s). */
void plasma_cuda_lag2s(cudaStream_t s, plasma_devstat_t *st, int call,
                       plasma_desc_t A, plasma_desc_t As, plasma_enum_t uplo);
void plasma_cuda_slag2d(cudaStream_t s, plasma_devstat_t *st,
                        plasma_desc_t As, plasma_desc_t A);
/* R <- B - A X with symmetric A given by its uplo triangle; then columnwise
 * max-abs of X and R into xnorm / rnorm (device). */
void plasma_cuda_residual(cudaStream_t s, plasma_devstat_t *st,
                          plasma_enum_t uplo, plasma_desc_t A,
                          plasma_desc_t B, plasma_desc_t X, plasma_desc_t R,
                          double *xnorm, double *rnorm);
/* X <- X + R (general descriptors of equal shape). */
void plasma_cuda_geadd(cudaStream_t s, plasma_devstat_t *st,
                       plasma_desc_t R, plasma_desc_t X);
/* B <- A (general descriptors of equal shape, same precision). */
void plasma_cuda_lacpy(cudaStream_t s, plasma_devstat_t *st,
                       plasma_desc_t A, plasma_desc_t B);

/* Tensor-core (tcgen05) trailing update of FP32 factors (cuda/update_tc.cu).
 * Product precisions: */
#define PLASMA_TC_TF32   1   /* one TF32 product                         */
#define PLASMA_TC_BF16   2   /* one BF16 product                         */
#define PLASMA_TC_TF32X3 3   /* lo*hi + hi*lo + hi*hi TF32 split (FP32)   */
#define PLASMA_TC_BF16X6 4   /* six products of a three-part BF16 split
                                (FP32; 256-wide tiles)                     */
int plasma_cuda_update_tc_ok(plasma_desc_t A, plasma_enum_t uplo);
/* Operand copies of the panels: full = 0 holds one panel (the caller
 * alternates two buffers), full = 1 every panel of the factor, so that an
 * update may lag any number of steps behind the panel stream. */
size_t plasma_cuda_panel_bytes(int tc_mode, plasma_desc_t A, int full);
int plasma_cuda_update_tc(cudaStream_t s, plasma_devstat_t *st, int tc_mode,
                          plasma_desc_t A, int k, int nlo, int nhi,
                          const void *panel, int full, int num_sms);
/* Copy of panel k in the operand format of tc_mode, in the layout `full`
 * (row tile m of the panel at tile m, or at k*mt - k(k-1)/2 + m - k; the
 * further parts of a split at one plane further each). */
void plasma_cuda_panel_round(cudaStream_t s, plasma_devstat_t *st, int tc_mode,
                             plasma_desc_t A, int k, void *panel, int full);
/* FP32 diagonal tile held in shared memory (order a multiple of 32, at most
 * 256); 0 when not applicable. */
int plasma_cuda_potrf_diag_smem(cudaStream_t s, plasma_devstat_t *st, int call,
                                plasma_enum_t uplo, plasma_desc_t A, int k,
                                int iinfo, int split);
/* FP32 panel kernels: 3 = FP32-accurate split TF32 products, 1 = TF32. */
void plasma_cuda_panel_set_split(int split);
/* A(i,i) = value for i in [i0, i1) (identity padding of FP32 factors). */
void plasma_cuda_set_diag(cudaStream_t s, plasma_desc_t A, int i0, int i1,
                          double value);

/* A view of a tile descriptor for the adjoint kernels (cuda/adjoint.cu):
 * logical element (i, j) is D(r0 + i, c0 + j), or D(r0 + j, c0 + i) when
 * trans; tri = 1 (2) reads entries above (below) the diagonal of the
 * untransposed view as zero; diag_scale = 1 halves its diagonal. */
typedef struct {
    plasma_desc_t D;
    int r0, c0;
    int trans;
    int tri;
    int diag_scale;
} plasma_view_t;

/* C = beta C + alpha op(A) op(B) (M x N, inner K); C is written inside the
 * mask ctri (0 all, 1 i >= j, 2 i <= j), outside it zeroed when czero. */
void plasma_cuda_gemm_view(cudaStream_t s, plasma_devstat_t *st, int M, int N,
                           int K, double alpha, plasma_view_t A, plasma_view_t B,
                           double beta, plasma_view_t C, int ctri, int czero);
/* dst(i,j) = op(src)(i,j) (masks and diagonal scale of src applied),
 * i < M, j < N. */
void plasma_cuda_copy_view(cudaStream_t s, plasma_devstat_t *st, int M, int N,
                           plasma_view_t src, plasma_view_t dst);
/* dst(i,j) = (src(i,j) + src(j,i)) / 2 for the n x n views. */
void plasma_cuda_symmetrize(cudaStream_t s, plasma_devstat_t *st, int n,
                            plasma_view_t src, plasma_view_t dst);

/* Refinement kernels (cuda/symv.cu, trsv.cu, vec.cu). */
size_t plasma_cuda_symv_work(plasma_desc_t A);
int plasma_cuda_symv(cudaStream_t s, plasma_devstat_t *st, plasma_enum_t uplo,
                     plasma_desc_t A, const double *x, const double *b,
                     double *r, double *xnorm, double *rnorm, double *work);
int plasma_cuda_trsv_block(plasma_desc_t A);
size_t plasma_cuda_trsv_sync_bytes(int nblk);
size_t plasma_cuda_trsv_w_bytes(plasma_desc_t A);
size_t plasma_cuda_trsv_scratch_bytes(plasma_desc_t A);
void plasma_cuda_trtri_blocks(cudaStream_t s, plasma_devstat_t *st,
                              plasma_enum_t uplo, plasma_desc_t A, void *W);
int plasma_cuda_trsv(cudaStream_t s, plasma_devstat_t *st, plasma_enum_t uplo,
                     int backward, plasma_desc_t A, const void *W, void *vec,
                     void *sync, int epoch, int num_sms);
int plasma_cuda_trsm_rows(cudaStream_t s, plasma_devstat_t *st, plasma_enum_t uplo,
                          int backward, plasma_desc_t A, const void *W, plasma_desc_t B,
                          int c0, int ncols, void *sync, int epoch, int num_sms);
size_t plasma_cuda_dots_work(int nv);
void plasma_cuda_dots(cudaStream_t s, const double *V, size_t ldv, int nv,
                      const double *w, size_t n, double *out, double *work);
void plasma_cuda_sub_combo(cudaStream_t s, const double *V, size_t ldv, int nv,
                           const double *h, double *w, size_t n);
void plasma_cuda_axpby(cudaStream_t s, double alpha, const double *x, double *y,
                       size_t n, int accumulate);
void plasma_cuda_combo(cudaStream_t s, const double *V, size_t ldv, int nv,
                       const double *c, double *y, size_t n, int accumulate);
void plasma_cuda_d2s(cudaStream_t s, const double *x, const double *sc,
                     float *y, size_t n, size_t npad, plasma_devstat_t *st,
                     int call);
void plasma_cuda_s2d(cudaStream_t s, const float *x, const double *sc,
                     double *y, size_t n);
/* d = 1/sqrt(diag(A)) (1 on the padding) and As <- D As D + shift I: the
 * diagonal scaling and shift of a low-precision factor's operand. */
void plasma_cuda_diag_rsqrt(cudaStream_t s, plasma_desc_t A, double *d,
                            size_t n, size_t npad);
void plasma_cuda_scale_shift(cudaStream_t s, plasma_desc_t As, int uplo,
                             const double *d, float shift);
void plasma_cuda_column(cudaStream_t s, plasma_desc_t D, int j, void *v,
                        int to_vec);
/* One-launch sweep with the context's ready-flag buffer (W from
 * plasma_cuda_trtri_blocks); returns 0 when the factor is not eligible. */
int plasma_sweep_reserve(plasma_context_t *plasma, plasma_desc_t A);
int plasma_sweep_rows(plasma_context_t *plasma, plasma_enum_t uplo, int backward,
                      plasma_desc_t A, const void *W, plasma_desc_t B, int c0, int ncols);
int plasma_desc_kept(plasma_context_t *c, int slot, plasma_enum_t precision,
                     plasma_enum_t type, int nb, int m, int n, plasma_desc_t *A);
int plasma_sweep(plasma_context_t *plasma, plasma_enum_t uplo, int backward,
                 plasma_desc_t A, const void *W, void *vec);

/* Host-side DAG walkers (compute/).  mode selects the trailing update of
 * FP32 factors: 0 or PlasmaFactorFP32 = FP32 arithmetic, PlasmaFactorTF32 /
 * PlasmaFactorBF16 = tensor-core products accumulated in FP32. */
void plasma_pXpotrf(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_sequence_t *sequence,
                    plasma_request_t *request, int call);
void plasma_pXpotrf_mode(plasma_context_t *plasma, plasma_enum_t uplo,
                         plasma_desc_t A, plasma_sequence_t *sequence,
                         plasma_request_t *request, int call, int mode);
/* The same factorization of a matrix whose tile columns are still arriving:
 * group g = tile columns [gstart[g], gstart[g+1]) is in place once event
 * arrive[g] has completed (gstart[0] = 0, gstart[ngroups] = A.nt,
 * 1 <= ngroups <= PLASMA_MAX_GROUPS). */
/* Grows the panel-copy scratch of plasma_pXpotrf_arrivals beforehand (a
 * slot that grows waits for every stream). */
void plasma_pXpotrf_reserve(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                            int mode, int full);
void plasma_pXpotrf_arrivals(plasma_context_t *plasma, plasma_enum_t uplo,
                             plasma_desc_t A, plasma_sequence_t *sequence,
                             plasma_request_t *request, int call, int mode,
                             int ngroups, const int *gstart, const cudaEvent_t *arrive);
void plasma_pXpotrs(plasma_context_t *plasma, plasma_enum_t uplo,
                    plasma_desc_t A, plasma_desc_t B,
                    plasma_sequence_t *sequence, plasma_request_t *request);
/* LU with partial pivoting (cuda/getrf.cu): the panel of tile column k
 * (pivots into ipiv, 1-based global rows; a zero pivot records info =
 * row + 1 and ends the walk; two launches per column), the interchanges of rows [j0, j1) on columns
 * [c0, c1), the inverses of the unit-lower and upper parts of diagonal tiles
 * [k0, k1) (nb x nb each at W + k*nb*nb), ||A||_inf of a general matrix and
 * the columnwise max |.| of an n x nrhs matrix (device doubles). */
void plasma_cuda_getrf_panel(cudaStream_t s, plasma_devstat_t *st, int call,
                             plasma_desc_t A, int k, int *ipiv, void *parts);
/* bytes of the `parts` workspace of plasma_cuda_getrf_panel for A */
size_t plasma_cuda_getrf_parts_bytes(plasma_desc_t A);
void plasma_cuda_laswp(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                       const int *ipiv, int j0, int j1, int c0, int c1);
void plasma_cuda_laswp_skip(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                            const int *ipiv, int j0, int j1, int c0, int c1, int skip0,
                            int skip1);
void plasma_cuda_trtri_lu(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                          int k0, int k1, void *WL, void *WU);
/* ||A||_inf and y -= A x (one right-hand side) of a general tile matrix;
 * part: scratch of plasma_cuda_gemv_part_bytes(A) bytes. */
size_t plasma_cuda_gemv_part_bytes(plasma_desc_t A);
/* LU trailing update A(m,n) -= A(m,k) A(k,n), m, n > k, for 64 x 64 FP32
 * tiles on the tensor cores; 0 (nothing launched) for other tilings. */
int plasma_cuda_lu_update(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A, int k);
/* LU block row A(k,n) <- WL_k A(k,n), n > k, for 64 x 64 FP32 tiles. */
int plasma_cuda_lu_rowsolve(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A, int k,
                            const void *WL);
/* The LU's interchanges composed into one permutation, and applied to one
 * column; 0 (nothing launched) when n is too large for one CTA. */
int plasma_cuda_lu_perm(cudaStream_t s, plasma_devstat_t *st, const int *ipiv, int n,
                        int *perm);
int plasma_cuda_permute_vec(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D, int col,
                            const int *perm, int n);
/* Largest panel height that the one-launch LU panel takes (64-wide tiles). */
int plasma_cuda_getrf_cluster_rows(int precision);
void plasma_cuda_lange_inf(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                           double *dnorm, double *part);
void plasma_cuda_gemv_sub(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t A,
                          const void *x, void *y, double *part);
void plasma_cuda_colmax(cudaStream_t s, plasma_devstat_t *st, plasma_desc_t D,
                        double *out);

/* Band Cholesky and the band solves on a band descriptor (compute/pbtrf.c). */
void plasma_pXpbtrf(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                    plasma_sequence_t *sequence, plasma_request_t *request, int call);
void plasma_pXpbtrs(plasma_context_t *plasma, plasma_enum_t uplo, plasma_desc_t A,
                    plasma_desc_t B, plasma_sequence_t *sequence, plasma_request_t *request);
void plasma_tune_trsm(plasma_context_t *plasma, plasma_enum_t dtyp, int m, int n);
void plasma_tune_pbtrf(plasma_context_t *plasma, plasma_enum_t dtyp, int n, int kd);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_B200_INTERNAL_H */
