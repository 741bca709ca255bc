/*
 * core_blas_impl.h -- precision-generic body of libplasma_core_blas.so, the
 * CPU tile kernels of the reference's kernel-substitution interface
 * (include/plasma_core_blas_z.h, plasma_core_blas_zc.h).  Included by
 * core_blas.c once with REAL = double, X(name) = plasma_core_d##name,
 * OMPX(name) = plasma_core_omp_d##name, and once with REAL = float and the
 * s names.
 *
 * These are host-memory kernels with the semantics of the BLAS / LAPACK
 * routines the reference calls through CBLAS / LAPACKE
 * (core_blas/core_zpotrf.c:54-63, core_ztrsm.c:87-100, core_zsyrk.c,
 * core_zgemm.c:89-102, core_zsymm.c, core_zlacpy.c:60-107,
 * core_zgeadd.c:74-163, core_zlansy.c, core_zlange.c), written from the
 * published reference-BLAS and LAPACK algorithms (dpotf2, dtrsm, dsyrk,
 * dgemm, dsymm, dlacpy, dlange, dlansy).  libplasma_b200.so never calls them:
 * its tile steps are whole-step GPU kernels.
 */

/* op(A)(i, j) of a column-major array */
#define OPA(P, ld, tr, i, j) ((tr) ? (P)[(size_t)(i) * (ld) + (j)] : (P)[(size_t)(j) * (ld) + (i)])

int X(potrf)(plasma_enum_t uplo, int n, REAL *A, int lda)
{
    if (uplo != PlasmaUpper && uplo != PlasmaLower) return -1;
    if (n < 0) return -2;
    if (lda < (n > 1 ? n : 1)) return -4;
#define AE(i, j) A[(size_t)(j) * lda + (i)]
    for (int j = 0; j < n; j++) {
        REAL ajj = AE(j, j);
        if (uplo == PlasmaLower)
            for (int k = 0; k < j; k++) ajj -= AE(j, k) * AE(j, k);
        else
            for (int k = 0; k < j; k++) ajj -= AE(k, j) * AE(k, j);
        if (!(ajj > 0)) {
            AE(j, j) = ajj;
            return j + 1;
        }
        ajj = (REAL)sqrt((double)ajj);
        AE(j, j) = ajj;
        const REAL r = (REAL)1 / ajj;
        if (uplo == PlasmaLower) {
            for (int i = j + 1; i < n; i++) {
                REAL s = AE(i, j);
                for (int k = 0; k < j; k++) s -= AE(i, k) * AE(j, k);
                AE(i, j) = s * r;
            }
        } else {
            for (int c = j + 1; c < n; c++) {
                REAL s = AE(j, c);
                for (int k = 0; k < j; k++) s -= AE(k, j) * AE(k, c);
                AE(j, c) = s * r;
            }
        }
    }
#undef AE
    return 0;
}

/* B <- alpha op(A)^-1 B (Left) or alpha B op(A)^-1 (Right), A triangular */
void X(trsm)(plasma_enum_t side, plasma_enum_t uplo, plasma_enum_t transa,
             plasma_enum_t diag, int m, int n, REAL alpha, const REAL *A, int lda,
             REAL *B, int ldb)
{
    const int tr = transa != PlasmaNoTrans;
    const int unit = diag == PlasmaUnit;
    /* op(A) is lower when (uplo lower, no transpose) or (upper, transpose) */
    const int lower = (uplo == PlasmaLower) != tr;
#define BE(i, j) B[(size_t)(j) * ldb + (i)]
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) BE(i, j) *= alpha;
    if (side == PlasmaLeft) {
        /* op(A) X = B, column by column of B */
        for (int j = 0; j < n; j++) {
            if (lower) {
                for (int i = 0; i < m; i++) {
                    REAL s = BE(i, j);
                    for (int l = 0; l < i; l++) s -= OPA(A, lda, tr, i, l) * BE(l, j);
                    BE(i, j) = unit ? s : s / OPA(A, lda, tr, i, i);
                }
            } else {
                for (int i = m - 1; i >= 0; i--) {
                    REAL s = BE(i, j);
                    for (int l = i + 1; l < m; l++) s -= OPA(A, lda, tr, i, l) * BE(l, j);
                    BE(i, j) = unit ? s : s / OPA(A, lda, tr, i, i);
                }
            }
        }
    } else {
        /* X op(A) = B, row by row of B: x op(A) = b */
        for (int i = 0; i < m; i++) {
            if (lower) {
                /* x_j depends on x_l, l > j */
                for (int j = n - 1; j >= 0; j--) {
                    REAL s = BE(i, j);
                    for (int l = j + 1; l < n; l++) s -= BE(i, l) * OPA(A, lda, tr, l, j);
                    BE(i, j) = unit ? s : s / OPA(A, lda, tr, j, j);
                }
            } else {
                for (int j = 0; j < n; j++) {
                    REAL s = BE(i, j);
                    for (int l = 0; l < j; l++) s -= BE(i, l) * OPA(A, lda, tr, l, j);
                    BE(i, j) = unit ? s : s / OPA(A, lda, tr, j, j);
                }
            }
        }
    }
#undef BE
}

/* C <- alpha op(A) op(A)^T + beta C on the uplo triangle; op(A) is n x k */
void X(syrk)(plasma_enum_t uplo, plasma_enum_t trans, int n, int k, REAL alpha,
             const REAL *A, int lda, REAL beta, REAL *C, int ldc)
{
    const int tr = trans != PlasmaNoTrans;
    for (int j = 0; j < n; j++) {
        const int i0 = uplo == PlasmaLower ? j : 0, i1 = uplo == PlasmaLower ? n : j + 1;
        for (int i = i0; i < i1; i++) {
            REAL s = 0;
            for (int l = 0; l < k; l++) s += OPA(A, lda, tr, i, l) * OPA(A, lda, tr, j, l);
            REAL *c = &C[(size_t)j * ldc + i];
            *c = (beta == (REAL)0 ? (REAL)0 : beta * *c) + alpha * s;
        }
    }
}

/* C <- alpha op(A) op(B) + beta C */
void X(gemm)(plasma_enum_t transa, plasma_enum_t transb, int m, int n, int k, REAL alpha,
             const REAL *A, int lda, const REAL *B, int ldb, REAL beta, REAL *C, int ldc)
{
    const int ta = transa != PlasmaNoTrans, tb = transb != PlasmaNoTrans;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            REAL s = 0;
            for (int l = 0; l < k; l++) s += OPA(A, lda, ta, i, l) * OPA(B, ldb, tb, l, j);
            REAL *c = &C[(size_t)j * ldc + i];
            *c = (beta == (REAL)0 ? (REAL)0 : beta * *c) + alpha * s;
        }
}

/* element (i, j) of the symmetric matrix stored in the uplo triangle of A */
static REAL X(sym_at)(plasma_enum_t uplo, const REAL *A, int lda, int i, int j)
{
    const int swap = uplo == PlasmaLower ? i < j : i > j;
    return swap ? A[(size_t)i * lda + j] : A[(size_t)j * lda + i];
}

/* C <- alpha A B + beta C (Left) or alpha B A + beta C (Right), A symmetric */
void X(symm)(plasma_enum_t side, plasma_enum_t uplo, int m, int n, REAL alpha,
             const REAL *A, int lda, const REAL *B, int ldb, REAL beta, REAL *C, int ldc)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            REAL s = 0;
            if (side == PlasmaLeft)
                for (int l = 0; l < m; l++)
                    s += X(sym_at)(uplo, A, lda, i, l) * B[(size_t)j * ldb + l];
            else
                for (int l = 0; l < n; l++)
                    s += B[(size_t)l * ldb + i] * X(sym_at)(uplo, A, lda, l, j);
            REAL *c = &C[(size_t)j * ldc + i];
            *c = (beta == (REAL)0 ? (REAL)0 : beta * *c) + alpha * s;
        }
}

/* core_zlacpy.c:60-107: LAPACK dlacpy for NoTrans, else the (conjugate)
 * transposed copy of the uplo part, B(j, i) = A(i, j) */
void X(lacpy)(plasma_enum_t uplo, plasma_enum_t transa, int m, int n, const REAL *A,
              int lda, REAL *B, int ldb)
{
    if (transa == PlasmaNoTrans) {
        for (int j = 0; j < n; j++) {
            const int i0 = uplo == PlasmaLower ? j : 0;
            const int i1 = uplo == PlasmaUpper ? (j + 1 < m ? j + 1 : m) : m;
            for (int i = i0; i < i1; i++)
                B[(size_t)j * ldb + i] = A[(size_t)j * lda + i];
        }
        return;
    }
    if (uplo == PlasmaUpper) {
        for (int i = 0; i < (m < n ? m : n); i++)
            for (int j = i; j < n; j++)
                B[j + (size_t)i * ldb] = A[i + (size_t)j * lda];
    } else if (uplo == PlasmaLower) {
        /* the reference's bound j <= min(i, n) reads column n when i >= n;
         * the copy stays inside the matrix here */
        for (int i = 0; i < m; i++)
            for (int j = 0; j < (i + 1 < n ? i + 1 : n); j++)
                B[j + (size_t)i * ldb] = A[i + (size_t)j * lda];
    } else {
        for (int i = 0; i < m; i++)
            for (int j = 0; j < n; j++)
                B[j + (size_t)i * ldb] = A[i + (size_t)j * lda];
    }
}

/* core_zgeadd.c:74-163: B <- beta B + alpha op(A), argument codes as there */
int X(geadd)(plasma_enum_t transa, int m, int n, REAL alpha, const REAL *A, int lda,
             REAL beta, REAL *B, int ldb)
{
    if (transa != PlasmaNoTrans && transa != PlasmaTrans && transa != PlasmaConjTrans)
        return -1;
    if (m < 0) return -2;
    if (n < 0) return -3;
    if (A == NULL) return -5;
    if ((transa == PlasmaNoTrans && lda < (m > 1 ? m : 1) && m > 0) ||
        (transa != PlasmaNoTrans && lda < (n > 1 ? n : 1) && n > 0))
        return -6;
    if (B == NULL) return -8;
    if (ldb < (m > 1 ? m : 1) && m > 0) return -9;
    if (m == 0 || n == 0 || (alpha == (REAL)0 && beta == (REAL)1))
        return PlasmaSuccess;
    const int tr = transa != PlasmaNoTrans;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++)
            B[(size_t)ldb * j + i] = beta * B[(size_t)ldb * j + i] + alpha * OPA(A, lda, tr, i, j);
    return PlasmaSuccess;
}

/* dlange: max |a|, one norm (max column sum), inf norm (max row sum; work
 * holds m row sums), Frobenius norm */
void X(lange)(plasma_enum_t norm, int m, int n, const REAL *A, int lda, double *work,
              double *value)
{
    double v = 0;
    if (m == 0 || n == 0) { *value = 0; return; }
    if (norm == PlasmaMaxNorm) {
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) {
                double a = fabs((double)A[(size_t)j * lda + i]);
                if (a > v || a != a) v = a;
            }
    } else if (norm == PlasmaOneNorm) {
        for (int j = 0; j < n; j++) {
            double s = 0;
            for (int i = 0; i < m; i++) s += fabs((double)A[(size_t)j * lda + i]);
            if (s > v || s != s) v = s;
        }
    } else if (norm == PlasmaInfNorm) {
        for (int i = 0; i < m; i++) work[i] = 0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) work[i] += fabs((double)A[(size_t)j * lda + i]);
        for (int i = 0; i < m; i++) if (work[i] > v || work[i] != work[i]) v = work[i];
    } else if (norm == PlasmaFrobeniusNorm) {
        double s = 0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) {
                double a = (double)A[(size_t)j * lda + i];
                s += a * a;
            }
        v = sqrt(s);
    } else {
        v = 0;
    }
    *value = v;
}

/* dlansy on the uplo triangle: max, one = inf (the matrix is symmetric; work
 * holds n column sums), Frobenius */
void X(lansy)(plasma_enum_t norm, plasma_enum_t uplo, int n, const REAL *A, int lda,
              double *work, double *value)
{
    double v = 0;
    if (n == 0) { *value = 0; return; }
    if (norm == PlasmaOneNorm || norm == PlasmaInfNorm) {
        for (int i = 0; i < n; i++) work[i] = 0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                const int stored = uplo == PlasmaLower ? i >= j : i <= j;
                if (!stored) continue;
                const double a = fabs((double)A[(size_t)j * lda + i]);
                work[j] += a;
                if (i != j) work[i] += a;
            }
        for (int i = 0; i < n; i++) if (work[i] > v || work[i] != work[i]) v = work[i];
    } else if (norm == PlasmaMaxNorm || norm == PlasmaFrobeniusNorm) {
        double s = 0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                const int stored = uplo == PlasmaLower ? i >= j : i <= j;
                if (!stored) continue;
                const double a = fabs((double)A[(size_t)j * lda + i]);
                if (norm == PlasmaMaxNorm) {
                    if (a > v || a != a) v = a;
                } else {
                    s += (i == j ? 1.0 : 2.0) * a * a;
                }
            }
        if (norm == PlasmaFrobeniusNorm) v = sqrt(s);
    }
    *value = v;
}

/* core_dzamax.c:20-61, without the task: columnwise (n values) or rowwise
 * (m values) max |a| */
void OMPX(amax)(int colrow, int m, int n, const REAL *A, int lda, double *values,
                plasma_sequence_t *sequence, plasma_request_t *request)
{
    (void)request;
    if (sequence != NULL && sequence->status != PlasmaSuccess) return;
    if (colrow == PlasmaColumnwise) {
        for (int j = 0; j < n; j++) {
            double v = fabs((double)A[(size_t)lda * j]);
            for (int i = 1; i < m; i++) {
                const double t = fabs((double)A[(size_t)lda * j + i]);
                if (t > v) v = t;
            }
            values[j] = v;
        }
    } else {
        for (int i = 0; i < m; i++) values[i] = fabs((double)A[i]);
        for (int j = 1; j < n; j++)
            for (int i = 0; i < m; i++) {
                const double t = fabs((double)A[(size_t)lda * j + i]);
                if (t > values[i]) values[i] = t;
            }
    }
}

#undef OPA
