/*
 * oracle_impl.h -- precision-generic body of the CPU oracle (TEST
 * INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
 * baseline of bench.py as the checker, never by the product library).
 *
 * Included by plasma_oracle.c once with REAL=double, P(x)=d##x and once with
 * REAL=float, P(x)=s##x.  It restates, on its own tile storage, the
 * reference's algorithms:
 *   tile Cholesky        compute/pzpotrf.c:27-126
 *   tile triangular solve compute/pztrsm.c:113-177 (Left, Lower) and
 *                        :43-107 (Left, Upper)
 *   band tile Cholesky   compute/pzpbtrf.c:37-118, and the band solves
 *                        (compute/pztbsm.c) as the tile solve cut to the band
 *   LU with partial pivoting compute/pzgetrf.c:37-232 (panel kernel
 *                        core_blas/core_zgetrf.c), the solve of zgetrs.c
 *   the LAPACK/BLAS tile kernels the reference calls through CBLAS/LAPACKE
 *   (core_blas/core_zpotrf.c:54-63, core_ztrsm.c:87-100, core_zsyrk.c,
 *   core_zgemm.c:89-102), written out from the published LAPACK algorithms
 *   (dpotf2: unblocked Cholesky with the "ajj <= 0 or NaN" test; dtrsm,
 *   dsyrk, dgemm: the reference BLAS loop orders).
 * The tile DAG runs as OpenMP tasks with depend() on tile base pointers, as
 * in core_blas/core_zgemm.c:125-127.
 */

/* ---- tile storage: tiles[(m) + mt*(n)] each column-major, ld = rows ---- */
typedef struct {
    int n, nb, mt;
    REAL **t;
} P(tiles_t);

static int P(tile_rows)(const P(tiles_t) *T, int m)
{
    return m < T->mt - 1 ? T->nb : T->n - T->nb * (T->mt - 1);
}

static int P(tiles_alloc)(P(tiles_t) *T, int n, int nb, int ncols)
{
    T->n = n;
    T->nb = nb;
    T->mt = (n + nb - 1) / nb;
    int nt = (ncols + nb - 1) / nb;
    if (nt < 1) nt = 1;
    T->t = (REAL **)calloc((size_t)T->mt * nt, sizeof(REAL *));
    if (!T->t) return -1;
    for (int j = 0; j < nt; j++)
        for (int i = 0; i < T->mt; i++) {
            int r = P(tile_rows)(T, i);
            int c = j < nt - 1 ? nb : ncols - nb * (nt - 1);
            if (c <= 0) c = 1;
            T->t[i + (size_t)T->mt * j] = (REAL *)calloc((size_t)r * c, sizeof(REAL));
        }
    return 0;
}

static void P(tiles_free)(P(tiles_t) *T, int ncols)
{
    int nt = (ncols + T->nb - 1) / T->nb;
    if (nt < 1) nt = 1;
    for (size_t i = 0; i < (size_t)T->mt * nt; i++) free(T->t[i]);
    free(T->t);
}

#define TL(T, m, n) ((T)->t[(m) + (size_t)(T)->mt * (n)])

static void P(to_tiles)(P(tiles_t) *T, const REAL *A, int lda, int ncols)
{
    int nb = T->nb;
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < T->n; i++) {
            int m = i / nb, k = j / nb;
            TL(T, m, k)[(size_t)(j - k * nb) * P(tile_rows)(T, m) + (i - m * nb)] =
                A[(size_t)j * lda + i];
        }
}

static void P(from_tiles)(const P(tiles_t) *T, REAL *A, int lda, int ncols,
                          int uplo)
{
    int nb = T->nb;
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < T->n; i++) {
            int m = i / nb, k = j / nb;
            /* full diagonal tiles are copied, as the reference's desc2tr does */
            if (uplo == ORACLE_LOWER && m < k) continue;
            if (uplo == ORACLE_UPPER && m > k) continue;
            A[(size_t)j * lda + i] =
                TL(T, m, k)[(size_t)(j - k * nb) * P(tile_rows)(T, m) + (i - m * nb)];
        }
}

/* ---------------- tile kernels (LAPACK / reference BLAS algorithms) ------ */

/* dpotf2, lower: A = L L^T; returns 0 or the failing column (1-based) */
static int P(k_potrf_lower)(int n, REAL *A, int lda)
{
    for (int j = 0; j < n; j++) {
        REAL ajj = A[j + (size_t)j * lda];
        for (int k = 0; k < j; k++)
            ajj -= A[j + (size_t)k * lda] * A[j + (size_t)k * lda];
        if (!(ajj > 0)) {
            A[j + (size_t)j * lda] = ajj;
            return j + 1;
        }
        ajj = (REAL)sqrt((double)ajj);
        A[j + (size_t)j * lda] = ajj;
        /* A(j+1:n, j) -= A(j+1:n, 0:j) * A(j, 0:j)^T ; then scale */
        for (int k = 0; k < j; k++) {
            REAL ajk = A[j + (size_t)k * lda];
            for (int i = j + 1; i < n; i++)
                A[i + (size_t)j * lda] -= A[i + (size_t)k * lda] * ajk;
        }
        REAL r = (REAL)1 / ajj;
        for (int i = j + 1; i < n; i++)
            A[i + (size_t)j * lda] *= r;
    }
    return 0;
}

/* dpotf2, upper: A = U^T U */
static int P(k_potrf_upper)(int n, REAL *A, int lda)
{
    for (int j = 0; j < n; j++) {
        REAL ajj = A[j + (size_t)j * lda];
        for (int k = 0; k < j; k++)
            ajj -= A[k + (size_t)j * lda] * A[k + (size_t)j * lda];
        if (!(ajj > 0)) {
            A[j + (size_t)j * lda] = ajj;
            return j + 1;
        }
        ajj = (REAL)sqrt((double)ajj);
        A[j + (size_t)j * lda] = ajj;
        REAL r = (REAL)1 / ajj;
        for (int c = j + 1; c < n; c++) {
            REAL s = A[j + (size_t)c * lda];
            for (int k = 0; k < j; k++)
                s -= A[k + (size_t)j * lda] * A[k + (size_t)c * lda];
            A[j + (size_t)c * lda] = s * r;
        }
    }
    return 0;
}

/* B(m x n) <- B * L^{-T}, L lower n x n (Right, Lower, Trans, NonUnit) */
static void P(k_trsm_rlt)(int m, int n, const REAL *L, int ldl, REAL *B, int ldb)
{
    for (int k = 0; k < n; k++) {
        REAL r = (REAL)1 / L[k + (size_t)k * ldl];
        for (int i = 0; i < m; i++) B[i + (size_t)k * ldb] *= r;
        for (int j = k + 1; j < n; j++) {
            REAL ljk = L[j + (size_t)k * ldl];
            if (ljk != 0)
                for (int i = 0; i < m; i++)
                    B[i + (size_t)j * ldb] -= ljk * B[i + (size_t)k * ldb];
        }
    }
}

/* B(m x n) <- U^{-T} B, U upper m x m (Left, Upper, Trans, NonUnit) */
static void P(k_trsm_lut)(int m, int n, const REAL *U, int ldu, REAL *B, int ldb)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            REAL s = B[i + (size_t)j * ldb];
            for (int k = 0; k < i; k++)
                s -= U[k + (size_t)i * ldu] * B[k + (size_t)j * ldb];
            B[i + (size_t)j * ldb] = s / U[i + (size_t)i * ldu];
        }
}

/* B <- L^{-1} B (Left, Lower, NoTrans) */
static void P(k_trsm_lln)(int m, int n, const REAL *L, int ldl, REAL *B, int ldb)
{
    for (int j = 0; j < n; j++)
        for (int k = 0; k < m; k++) {
            REAL bk = B[k + (size_t)j * ldb] / L[k + (size_t)k * ldl];
            B[k + (size_t)j * ldb] = bk;
            for (int i = k + 1; i < m; i++)
                B[i + (size_t)j * ldb] -= bk * L[i + (size_t)k * ldl];
        }
}

/* B <- L^{-T} B (Left, Lower, Trans) */
static void P(k_trsm_llt)(int m, int n, const REAL *L, int ldl, REAL *B, int ldb)
{
    for (int j = 0; j < n; j++)
        for (int i = m - 1; i >= 0; i--) {
            REAL s = B[i + (size_t)j * ldb];
            for (int k = i + 1; k < m; k++)
                s -= L[k + (size_t)i * ldl] * B[k + (size_t)j * ldb];
            B[i + (size_t)j * ldb] = s / L[i + (size_t)i * ldl];
        }
}

/* B <- U^{-1} B (Left, Upper, NoTrans) */
static void P(k_trsm_lun)(int m, int n, const REAL *U, int ldu, REAL *B, int ldb)
{
    for (int j = 0; j < n; j++)
        for (int k = m - 1; k >= 0; k--) {
            REAL bk = B[k + (size_t)j * ldb] / U[k + (size_t)k * ldu];
            B[k + (size_t)j * ldb] = bk;
            for (int i = 0; i < k; i++)
                B[i + (size_t)j * ldb] -= bk * U[i + (size_t)k * ldu];
        }
}

/* C(m x n) -= A(m x k) B(n x k)^T ; lower_only restricts to i >= j */
static void P(k_gemm_nt)(int m, int n, int k, const REAL *A, int lda,
                         const REAL *B, int ldb, REAL *C, int ldc, int lower_only)
{
    for (int j = 0; j < n; j++) {
        int i0 = lower_only ? j : 0;
        REAL *c = C + (size_t)j * ldc;
        int l = 0;
        for (; l + 4 <= k; l += 4) {
            REAL b0 = B[j + (size_t)l * ldb], b1 = B[j + (size_t)(l + 1) * ldb];
            REAL b2 = B[j + (size_t)(l + 2) * ldb], b3 = B[j + (size_t)(l + 3) * ldb];
            const REAL *a0 = A + (size_t)l * lda, *a1 = a0 + lda;
            const REAL *a2 = a1 + lda, *a3 = a2 + lda;
            for (int i = i0; i < m; i++)
                c[i] -= a0[i] * b0 + a1[i] * b1 + a2[i] * b2 + a3[i] * b3;
        }
        for (; l < k; l++) {
            REAL b0 = B[j + (size_t)l * ldb];
            const REAL *a0 = A + (size_t)l * lda;
            for (int i = i0; i < m; i++) c[i] -= a0[i] * b0;
        }
    }
}

/* C(m x n) -= A(k x m)^T B(k x n) ; upper_only restricts to i <= j */
static void P(k_gemm_tn)(int m, int n, int k, const REAL *A, int lda,
                         const REAL *B, int ldb, REAL *C, int ldc, int upper_only)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < (upper_only ? (j + 1 < m ? j + 1 : m) : m); i++) {
            REAL s = 0;
            const REAL *a = A + (size_t)i * lda, *b = B + (size_t)j * ldb;
            for (int l = 0; l < k; l++) s += a[l] * b[l];
            C[i + (size_t)j * ldc] -= s;
        }
}

/* C(m x n) -= A(m x k) B(k x n) */
static void P(k_gemm_nn)(int m, int n, int k, const REAL *A, int lda,
                         const REAL *B, int ldb, REAL *C, int ldc)
{
    for (int j = 0; j < n; j++)
        for (int l = 0; l < k; l++) {
            REAL b = B[l + (size_t)j * ldb];
            const REAL *a = A + (size_t)l * lda;
            REAL *c = C + (size_t)j * ldc;
            for (int i = 0; i < m; i++) c[i] -= a[i] * b;
        }
}

/* ---------------- parallel tile algorithms ------------------------------ */

/* compute/pzpotrf.c:27-126 ; returns info (nb*k + local) or 0 */
static int P(p_potrf)(P(tiles_t) *A, int uplo)
{
    int info = 0;
    const int mt = A->mt, nb = A->nb;
    #pragma omp parallel
    #pragma omp master
    {
        for (int k = 0; k < mt; k++) {
            REAL *akk = TL(A, k, k);
            int nk = P(tile_rows)(A, k);
            #pragma omp task depend(inout: akk[0]) shared(info)
            {
                int st;
                #pragma omp atomic read
                st = info;
                if (st == 0) {
                    int i = uplo == ORACLE_LOWER ? P(k_potrf_lower)(nk, akk, nk)
                                                 : P(k_potrf_upper)(nk, akk, nk);
                    if (i != 0) {
                        #pragma omp critical (oracle_info)
                        if (info == 0) info = nb * k + i;
                    }
                }
            }
            for (int m = k + 1; m < mt; m++) {
                int nm = P(tile_rows)(A, m);
                if (uplo == ORACLE_LOWER) {
                    REAL *amk = TL(A, m, k);
                    #pragma omp task depend(in: akk[0]) depend(inout: amk[0]) shared(info)
                    if (info == 0) P(k_trsm_rlt)(nm, nk, akk, nk, amk, nm);
                } else {
                    REAL *akm = TL(A, k, m);
                    #pragma omp task depend(in: akk[0]) depend(inout: akm[0]) shared(info)
                    if (info == 0) P(k_trsm_lut)(nk, nm, akk, nk, akm, nk);
                }
            }
            for (int m = k + 1; m < mt; m++) {
                int nm = P(tile_rows)(A, m);
                for (int n = k + 1; n <= m; n++) {
                    int nn = P(tile_rows)(A, n);
                    if (uplo == ORACLE_LOWER) {
                        REAL *amk = TL(A, m, k), *ank = TL(A, n, k), *amn = TL(A, m, n);
                        #pragma omp task depend(in: amk[0], ank[0]) depend(inout: amn[0]) shared(info)
                        if (info == 0)
                            P(k_gemm_nt)(nm, nn, nk, amk, nm, ank, nn, amn, nm, m == n);
                    } else {
                        /* A(n,m) -= A(k,n)^T A(k,m) */
                        REAL *akn = TL(A, k, n), *akm = TL(A, k, m), *anm = TL(A, n, m);
                        #pragma omp task depend(in: akn[0], akm[0]) depend(inout: anm[0]) shared(info)
                        if (info == 0)
                            P(k_gemm_tn)(nn, nm, nk, akn, nk, akm, nk, anm, nn, m == n);
                    }
                }
            }
        }
    }
    return info;
}

/* compute/pztrsm.c (Left): trans = 0 solves op = L (or U^T), 1 solves L^T (or U)
 * B is n x nrhs in tiles (B->mt row tiles, one column block per nb cols).
 * kt > 0: the factor is a band of kt tiles per tile column (diagonal
 * included), and only those tiles are visited, as in the reference's band
 * solve compute/pztbsm.c. */
static void P(p_trsm)(P(tiles_t) *A, P(tiles_t) *B, int nrhs, int uplo, int second,
                      int kt)
{
    const int mt = A->mt, nb = A->nb;
    const int nt = (nrhs + nb - 1) / nb;
    #pragma omp parallel
    #pragma omp master
    for (int step = 0; step < mt; step++) {
        /* forward sweep for (Lower,NoTrans) and (Upper,Trans); backward else */
        int k = second ? mt - 1 - step : step;
        int nk = P(tile_rows)(A, k);
        REAL *akk = TL(A, k, k);
        for (int n = 0; n < nt; n++) {
            int nc = n < nt - 1 ? nb : nrhs - nb * (nt - 1);
            REAL *bkn = TL(B, k, n);
            #pragma omp task depend(in: akk[0]) depend(inout: bkn[0])
            {
                if (uplo == ORACLE_LOWER) {
                    if (!second) P(k_trsm_lln)(nk, nc, akk, nk, bkn, nk);
                    else         P(k_trsm_llt)(nk, nc, akk, nk, bkn, nk);
                } else {
                    if (!second) P(k_trsm_lut)(nk, nc, akk, nk, bkn, nk);
                    else         P(k_trsm_lun)(nk, nc, akk, nk, bkn, nk);
                }
            }
        }
        int mlo = second ? 0 : k + 1, mhi = second ? k : mt;
        if (kt > 0) {
            if (second) mlo = k - kt + 1 > 0 ? k - kt + 1 : 0;
            else        mhi = k + kt < mt ? k + kt : mt;
        }
        for (int m = mlo; m < mhi; m++) {
            int nm = P(tile_rows)(A, m);
            for (int n = 0; n < nt; n++) {
                int nc = n < nt - 1 ? nb : nrhs - nb * (nt - 1);
                REAL *bkn = TL(B, k, n), *bmn = TL(B, m, n);
                if (uplo == ORACLE_LOWER) {
                    if (!second) {        /* B(m) -= L(m,k) B(k) */
                        REAL *amk = TL(A, m, k);
                        #pragma omp task depend(in: amk[0], bkn[0]) depend(inout: bmn[0])
                        P(k_gemm_nn)(nm, nc, nk, amk, nm, bkn, nk, bmn, nm);
                    } else {              /* B(m) -= L(k,m)^T B(k) */
                        REAL *akm = TL(A, k, m);
                        #pragma omp task depend(in: akm[0], bkn[0]) depend(inout: bmn[0])
                        P(k_gemm_tn)(nm, nc, nk, akm, nk, bkn, nk, bmn, nm, 0);
                    }
                } else {
                    if (!second) {        /* B(m) -= U(k,m)^T B(k) */
                        REAL *akm = TL(A, k, m);
                        #pragma omp task depend(in: akm[0], bkn[0]) depend(inout: bmn[0])
                        P(k_gemm_tn)(nm, nc, nk, akm, nk, bkn, nk, bmn, nm, 0);
                    } else {              /* B(m) -= U(m,k) B(k) */
                        REAL *amk = TL(A, m, k);
                        #pragma omp task depend(in: amk[0], bkn[0]) depend(inout: bmn[0])
                        P(k_gemm_nn)(nm, nc, nk, amk, nm, bkn, nk, bmn, nm);
                    }
                }
            }
        }
    }
}

/* compute/pzpbtrf.c:37-118: the band tile loop.  For each k: POTRF of tile
 * (k,k); for the tiles m = k+1 .. k+kt-1 of the band below it (right of it
 * for upper storage): TRSM, SYRK on (m,m), GEMM on (m,n) for k < n < m.
 * Tiles outside the band are never visited.  Returns info as p_potrf. */
static int P(p_pbtrf)(P(tiles_t) *A, int uplo, int kt)
{
    int info = 0;
    const int mt = A->mt, nb = A->nb;
    #pragma omp parallel
    #pragma omp master
    {
        for (int k = 0; k < mt; k++) {
            REAL *akk = TL(A, k, k);
            int nk = P(tile_rows)(A, k);
            #pragma omp task depend(inout: akk[0]) shared(info)
            {
                int st;
                #pragma omp atomic read
                st = info;
                if (st == 0) {
                    int i = uplo == ORACLE_LOWER ? P(k_potrf_lower)(nk, akk, nk)
                                                 : P(k_potrf_upper)(nk, akk, nk);
                    if (i != 0) {
                        #pragma omp critical (oracle_info)
                        if (info == 0) info = nb * k + i;
                    }
                }
            }
            const int mhi = k + kt < mt ? k + kt : mt;
            for (int m = k + 1; m < mhi; m++) {
                int nm = P(tile_rows)(A, m);
                if (uplo == ORACLE_LOWER) {
                    REAL *amk = TL(A, m, k);
                    #pragma omp task depend(in: akk[0]) depend(inout: amk[0]) shared(info)
                    if (info == 0) P(k_trsm_rlt)(nm, nk, akk, nk, amk, nm);
                } else {
                    REAL *akm = TL(A, k, m);
                    #pragma omp task depend(in: akk[0]) depend(inout: akm[0]) shared(info)
                    if (info == 0) P(k_trsm_lut)(nk, nm, akk, nk, akm, nk);
                }
                for (int n = k + 1; n <= m; n++) {
                    int nn = P(tile_rows)(A, n);
                    if (uplo == ORACLE_LOWER) {
                        REAL *amk = TL(A, m, k), *ank = TL(A, n, k), *amn = TL(A, m, n);
                        #pragma omp task depend(in: amk[0], ank[0]) depend(inout: amn[0]) shared(info)
                        if (info == 0)
                            P(k_gemm_nt)(nm, nn, nk, amk, nm, ank, nn, amn, nm, m == n);
                    } else {
                        REAL *akn = TL(A, k, n), *akm = TL(A, k, m), *anm = TL(A, n, m);
                        #pragma omp task depend(in: akn[0], akm[0]) depend(inout: anm[0]) shared(info)
                        if (info == 0)
                            P(k_gemm_tn)(nn, nm, nk, akn, nk, akm, nk, anm, nn, m == n);
                    }
                }
            }
        }
    }
    return info;
}

/* LAPACK band storage <-> tiles of the n x n matrix (zero outside the band):
 * A(i,j) = AB[off + i - j + j*ldab], off = kd (upper) or 0 (lower), for
 * 0 <= i-j <= kd (lower) or 0 <= j-i <= kd (upper) -- the layout of
 * compute/pzpb2desc.c:20-22. */
static void P(band_to_tiles)(P(tiles_t) *T, int uplo, int kd, const REAL *AB, int ldab)
{
    const int n = T->n, nb = T->nb, off = uplo == ORACLE_UPPER ? kd : 0;
    for (int j = 0; j < n; j++) {
        int i0 = uplo == ORACLE_LOWER ? j : (j - kd > 0 ? j - kd : 0);
        int i1 = uplo == ORACLE_LOWER ? (j + kd < n - 1 ? j + kd : n - 1) : j;
        for (int i = i0; i <= i1; i++) {
            int m = i / nb, k = j / nb;
            TL(T, m, k)[(size_t)(j - k * nb) * P(tile_rows)(T, m) + (i - m * nb)] =
                AB[(size_t)j * ldab + off + i - j];
        }
    }
}

static void P(tiles_to_band)(const P(tiles_t) *T, int uplo, int kd, REAL *AB, int ldab)
{
    const int n = T->n, nb = T->nb, off = uplo == ORACLE_UPPER ? kd : 0;
    for (int j = 0; j < n; j++) {
        int i0 = uplo == ORACLE_LOWER ? j : (j - kd > 0 ? j - kd : 0);
        int i1 = uplo == ORACLE_LOWER ? (j + kd < n - 1 ? j + kd : n - 1) : j;
        for (int i = i0; i <= i1; i++) {
            int m = i / nb, k = j / nb;
            AB[(size_t)j * ldab + off + i - j] =
                TL(T, m, k)[(size_t)(j - k * nb) * P(tile_rows)(T, m) + (i - m * nb)];
        }
    }
}

/* ---------------- LU with partial pivoting ------------------------------ */

/* The reference's tile LU (compute/pzgetrf.c:37-232, panel kernel
 * core_blas/core_zgetrf.c:20-238) on column-major A (n x n, lda): for each
 * block column of width nb, the panel (all rows from the block's first row
 * down) is factored column by column -- pivot search over the whole panel
 * column (the first entry of largest magnitude, as LAPACK's idamax), row
 * interchange, the column divided by the pivot (multiplied by its reciprocal
 * when |pivot| < sfmin, core_zgetrf.c:125-145), rank-1 update of the panel's
 * other columns -- then the columns right of the panel get a unit-lower
 * solve on the block row and the GEMM update below it.  Interchanges are
 * applied to whole rows at once; the reference defers those left of the
 * panel to the end (:196-228), and interchanges move values without
 * arithmetic, so the factors are the same.  ipiv is 1-based, as LAPACK's.
 * Returns info = the first zero pivot (1-based); like the reference, whose
 * failed sequence skips every later task, the factorization stops at the
 * panel that holds it. */
static int P(p_getrf)(int n, REAL *A, int lda, int *ipiv, int nb)
{
#define GE(i, j) A[(size_t)(j) * lda + (i)]
    const REAL sfmin = sizeof(REAL) == 4 ? (REAL)FLT_MIN : (REAL)DBL_MIN;
    for (int k0 = 0; k0 < n; k0 += nb) {
        const int kb = n - k0 < nb ? n - k0 : nb;
        for (int j = k0; j < k0 + kb; j++) {
            int jp = j;
            REAL best = (REAL)fabs((double)GE(j, j));
            for (int i = j + 1; i < n; i++) {
                REAL v = (REAL)fabs((double)GE(i, j));
                if (v > best) { best = v; jp = i; }
            }
            ipiv[j] = jp + 1;
            if (best == (REAL)0)
                return j + 1;
            if (jp != j)
                for (int c = 0; c < n; c++) {
                    REAL t = GE(j, c); GE(j, c) = GE(jp, c); GE(jp, c) = t;
                }
            const REAL piv = GE(j, j);
            if ((REAL)fabs((double)piv) >= sfmin) {
                for (int i = j + 1; i < n; i++) GE(i, j) /= piv;
            } else {
                const REAL r = (REAL)1 / piv;
                for (int i = j + 1; i < n; i++) GE(i, j) *= r;
            }
            #pragma omp parallel for schedule(static)
            for (int c = j + 1; c < k0 + kb; c++) {
                const REAL u = GE(j, c);
                for (int i = j + 1; i < n; i++) GE(i, c) -= GE(i, j) * u;
            }
        }
        /* block row: unit-lower solve; below it: GEMM */
        #pragma omp parallel for schedule(dynamic, 4)
        for (int c = k0 + kb; c < n; c++) {
            for (int l = k0; l < k0 + kb; l++) {
                const REAL u = GE(l, c);
                for (int i = l + 1; i < k0 + kb; i++) GE(i, c) -= GE(i, l) * u;
            }
            for (int l = k0; l < k0 + kb; l++) {
                const REAL u = GE(l, c);
                for (int i = k0 + kb; i < n; i++) GE(i, c) -= GE(i, l) * u;
            }
        }
    }
    return 0;
#undef GE
}

/* plasma_getrs (compute/zgetrs.c): the interchanges on B (geswp), then the
 * unit-lower and the upper solves (pztrsm) */
static void P(p_getrs)(int n, int nrhs, const REAL *A, int lda, const int *ipiv,
                       REAL *B, int ldb)
{
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < nrhs; c++) {
        REAL *b = B + (size_t)c * ldb;
        for (int j = 0; j < n; j++) {
            int p = ipiv[j] - 1;
            if (p != j) { REAL t = b[j]; b[j] = b[p]; b[p] = t; }
        }
        for (int l = 0; l < n; l++) {
            const REAL u = b[l];
            const REAL *a = A + (size_t)l * lda;
            for (int i = l + 1; i < n; i++) b[i] -= a[i] * u;
        }
        for (int l = n - 1; l >= 0; l--) {
            const REAL *a = A + (size_t)l * lda;
            b[l] /= a[l];
            const REAL u = b[l];
            for (int i = 0; i < l; i++) b[i] -= a[i] * u;
        }
    }
}

int P(oracle_getrf)(int n, REAL *A, int lda, int *ipiv, int nb)
{
    if (n == 0) return 0;
    return P(p_getrf)(n, A, lda, ipiv, nb);
}

int P(oracle_getrs)(int n, int nrhs, const REAL *A, int lda, const int *ipiv,
                    REAL *B, int ldb)
{
    if (n == 0 || nrhs == 0) return 0;
    P(p_getrs)(n, nrhs, A, lda, ipiv, B, ldb);
    return 0;
}

int P(oracle_gesv)(int n, int nrhs, REAL *A, int lda, int *ipiv, REAL *B, int ldb,
                   int nb)
{
    if (n == 0 || nrhs == 0) return 0;
    int info = P(p_getrf)(n, A, lda, ipiv, nb);
    if (info == 0)
        P(p_getrs)(n, nrhs, A, lda, ipiv, B, ldb);
    return info;
}

/* ---------------- LAPACK-layout entry points ---------------------------- */

/* plasma_pbtrf (compute/zpbtrf.c): band tiles with kt = 1 + ceil(kd/nb), the
 * reference's klt/kut (control/descriptor.c:204-211); AB is left unchanged
 * when info > 0. */
int P(oracle_pbtrf)(int uplo, int n, int kd, REAL *AB, int ldab, int nb)
{
    if (n == 0) return 0;
    P(tiles_t) T;
    P(tiles_alloc)(&T, n, nb, n);
    P(band_to_tiles)(&T, uplo, kd, AB, ldab);
    int info = P(p_pbtrf)(&T, uplo, 1 + (kd + nb - 1) / nb);
    if (info == 0)
        P(tiles_to_band)(&T, uplo, kd, AB, ldab);
    P(tiles_free)(&T, n);
    return info;
}

/* plasma_pbtrs (compute/zpbtrs.c:280-294): the two band sweeps */
int P(oracle_pbtrs)(int uplo, int n, int kd, int nrhs, const REAL *AB, int ldab,
                    REAL *B, int ldb, int nb)
{
    if (n == 0 || nrhs == 0) return 0;
    P(tiles_t) TA, TB;
    P(tiles_alloc)(&TA, n, nb, n);
    P(tiles_alloc)(&TB, n, nb, nrhs);
    P(band_to_tiles)(&TA, uplo, kd, AB, ldab);
    P(to_tiles)(&TB, B, ldb, nrhs);
    const int kt = 1 + (kd + nb - 1) / nb;
    P(p_trsm)(&TA, &TB, nrhs, uplo, 0, kt);
    P(p_trsm)(&TA, &TB, nrhs, uplo, 1, kt);
    P(from_tiles)(&TB, B, ldb, nrhs, 0);
    P(tiles_free)(&TA, n);
    P(tiles_free)(&TB, nrhs);
    return 0;
}

int P(oracle_potrf)(int uplo, int n, REAL *A, int lda, int nb)
{
    if (n == 0) return 0;
    P(tiles_t) T;
    P(tiles_alloc)(&T, n, nb, n);
    P(to_tiles)(&T, A, lda, n);
    int info = P(p_potrf)(&T, uplo);
    if (info == 0)
        P(from_tiles)(&T, A, lda, n, uplo);
    P(tiles_free)(&T, n);
    return info;
}

int P(oracle_potrs)(int uplo, int n, int nrhs, const REAL *A, int lda,
                    REAL *B, int ldb, int nb)
{
    if (n == 0 || nrhs == 0) return 0;
    P(tiles_t) TA, TB;
    P(tiles_alloc)(&TA, n, nb, n);
    P(tiles_alloc)(&TB, n, nb, nrhs);
    P(to_tiles)(&TA, A, lda, n);
    P(to_tiles)(&TB, B, ldb, nrhs);
    P(p_trsm)(&TA, &TB, nrhs, uplo, 0, 0);
    P(p_trsm)(&TA, &TB, nrhs, uplo, 1, 0);
    P(from_tiles)(&TB, B, ldb, nrhs, 0);
    P(tiles_free)(&TA, n);
    P(tiles_free)(&TB, nrhs);
    return 0;
}

int P(oracle_posv)(int uplo, int n, int nrhs, REAL *A, int lda, REAL *B,
                   int ldb, int nb)
{
    if (n == 0 || nrhs == 0) return 0;
    P(tiles_t) TA, TB;
    P(tiles_alloc)(&TA, n, nb, n);
    P(tiles_alloc)(&TB, n, nb, nrhs);
    P(to_tiles)(&TA, A, lda, n);
    P(to_tiles)(&TB, B, ldb, nrhs);
    int info = P(p_potrf)(&TA, uplo);
    if (info == 0) {
        P(p_trsm)(&TA, &TB, nrhs, uplo, 0, 0);
        P(p_trsm)(&TA, &TB, nrhs, uplo, 1, 0);
        P(from_tiles)(&TA, A, lda, n, uplo);
        P(from_tiles)(&TB, B, ldb, nrhs, 0);
    }
    P(tiles_free)(&TA, n);
    P(tiles_free)(&TB, nrhs);
    return info;
}

/* Inverse of an SPD matrix from its Cholesky factor held in the uplo
 * triangle of A (compute/zpotri.c:228-235: plasma_pztrtri(uplo, NonUnit)
 * then plasma_pzlauum(uplo)), restated unblocked from the published LAPACK
 * algorithms the reference's tile kernels implement: dtrti2 (inverse of a
 * triangular matrix, column by column against the part already inverted)
 * and dlauu2 (L^T L, or U U^T, row by row).  Returns info = i + 1 when
 * A(i,i) is exactly zero (dtrtri), leaving A unchanged; the other triangle
 * is not touched. */
int P(oracle_potri)(int uplo, int n, REAL *A, int lda)
{
#define AE(i, j) A[(i) + (size_t)(j) * lda]
    for (int i = 0; i < n; i++)
        if (AE(i, i) == (REAL)0)
            return i + 1;
    REAL *x = (REAL *)malloc(sizeof(REAL) * (size_t)(n > 0 ? n : 1));
    if (uplo == ORACLE_LOWER) {
        /* dtrti2, lower: columns from the last one back */
        for (int j = n - 1; j >= 0; j--) {
            AE(j, j) = (REAL)1 / AE(j, j);
            const REAL ajj = -AE(j, j);
            /* A(j+1:n, j) = ajj * T(j+1:n, j+1:n) A(j+1:n, j), T lower */
            for (int i = j + 1; i < n; i++) x[i] = AE(i, j);
            for (int i = j + 1; i < n; i++) {
                REAL t = 0;
                for (int k = j + 1; k <= i; k++) t += AE(i, k) * x[k];
                AE(i, j) = ajj * t;
            }
        }
        /* dlauu2, lower: A <- L^T L */
        for (int i = 0; i < n; i++) {
            const REAL aii = AE(i, i);
            REAL d = 0;
            for (int k = i; k < n; k++) d += AE(k, i) * AE(k, i);
            /* A(i, 0:i) = aii A(i, 0:i) + A(i+1:n, 0:i)^T A(i+1:n, i) */
            for (int j = 0; j < i; j++) {
                REAL t = aii * AE(i, j);
                for (int k = i + 1; k < n; k++) t += AE(k, j) * AE(k, i);
                AE(i, j) = t;
            }
            AE(i, i) = d;
        }
    } else {
        /* dtrti2, upper: columns from the first one on */
        for (int j = 0; j < n; j++) {
            AE(j, j) = (REAL)1 / AE(j, j);
            const REAL ajj = -AE(j, j);
            /* A(0:j, j) = ajj * T(0:j, 0:j) A(0:j, j), T upper */
            for (int i = 0; i < j; i++) x[i] = AE(i, j);
            for (int i = 0; i < j; i++) {
                REAL t = 0;
                for (int k = i; k < j; k++) t += AE(i, k) * x[k];
                AE(i, j) = ajj * t;
            }
        }
        /* dlauu2, upper: A <- U U^T */
        for (int i = 0; i < n; i++) {
            const REAL aii = AE(i, i);
            REAL d = 0;
            for (int k = i; k < n; k++) d += AE(i, k) * AE(i, k);
            /* A(0:i, i) = aii A(0:i, i) + A(0:i, i+1:n) A(i, i+1:n)^T */
            for (int j = 0; j < i; j++) {
                REAL t = aii * AE(j, i);
                for (int k = i + 1; k < n; k++) t += AE(j, k) * AE(i, k);
                AE(j, i) = t;
            }
            AE(i, i) = d;
        }
    }
    free(x);
    return 0;
#undef AE
}

