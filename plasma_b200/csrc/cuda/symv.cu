// symv.cu -- FP64 symmetric matrix-vector product on tile storage:
//     r = b - A x      (A symmetric, held in one triangle of a descriptor)
// plus the max norms of x and r, i.e. one refinement residual of dsposv
// (pdlacpy B->R, pdsymm, pdamax: compute/zcposv.c:466-472,
// compute/pzsymm.c:29-211, compute/pdzamax.c:24-79) for one right-hand side.
//
// Each stored tile S = A(p,q) is read from HBM exactly once by one CTA, which
// forms both contributions  S x_q  (to rows of block p)  and  S^T x_p  (to
// rows of block q).  Lanes own rows, so every warp load is consecutive
// doubles of one column (16-byte loads of two rows per lane on the full
// off-diagonal tiles); the transposed product of a block is reduced across
// lanes by a butterfly (16 columns per warp pass; one CTA per SM keeps the
// loop in registers).  The per-tile partial vectors go to
// a workspace and a second kernel sums them in a fixed order, so results are
// bit-reproducible.
//
// The same pass with |a| and x = 1 gives the row sums of |A|, whose maximum
// is ||A||_inf (plasma_pdlansy, compute/pzlansy.c:83-131): one read of the
// stored triangle.
#include "common.cuh"

namespace {

constexpr int SV_THREADS = 256;

// v[i] summed over the 32 lanes, for 16 columns: lane l (and l + 16) ends
// up with the sum of column l & 15
__device__ __forceinline__ double butterfly16(double (&v)[16], int lane)
{
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i], 16);
#pragma unroll
    for (int off = 8; off >= 1; off >>= 1) {
        const bool hi = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < off; i++) {
            double send = hi ? v[i] : v[i + off];
            double keep = hi ? v[i + off] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    return v[0];
}

__device__ __forceinline__ void stored_tile(int t, int mt, int uplo, int &p, int &q)
{
    // column-major enumeration of the stored triangle of tiles
    q = 0;
    if (uplo == PlasmaLower) {
        while (t >= mt - q) { t -= mt - q; q++; }
        p = q + t;
    } else {
        while (t >= q + 1) { t -= q + 1; q++; }
        p = t;
    }
}

template <bool ABS>
__global__ void __launch_bounds__(SV_THREADS, 1)
k_symv_tiles(plasma_desc_t A, int uplo, const double *x, double *part,
             const plasma_devstat_t *st)
{
    __shared__ __align__(16) double xp_s[512];
    __shared__ double xq_s[512];
    __shared__ double ypart[8][512];
    if (plasma_failed(st)) return;
    const int mt = A.mt, nb = A.mb;
    int p, q;
    stored_tile(blockIdx.x, mt, uplo, p, q);
    const double *S = (const double *)plasma_tile_addr(A, p, q);
    const int ld = plasma_tile_mmain(A, p);
    const int rows = plasma_tile_mview(A, p);
    const int cols = plasma_tile_mview(A, q);
    const bool diag = p == q;
    const bool lower = uplo == PlasmaLower;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int i = tid; i < nb; i += SV_THREADS) {
        xp_s[i] = i < rows ? (ABS ? 1.0 : x[(size_t)p * nb + i]) : 0.0;
        xq_s[i] = i < cols ? (ABS ? 1.0 : x[(size_t)q * nb + i]) : 0.0;
    }
    for (int i = tid; i < 8 * 512; i += SV_THREADS) (&ypart[0][0])[i] = 0.0;
    __syncthreads();

    double *yq_out = part + ((size_t)q * mt + p) * nb;     // S^T x_p -> block q
    // Full off-diagonal tiles (all but mt of the mt(mt+1)/2): 16-byte loads,
    // lane l owns rows 2l and 2l+1 of each 64-row block, no predicates.
    const bool fast = !diag && rows == nb && cols == nb && nb % 64 == 0 && nb <= 512 &&
                      (ld & 1) == 0 && ((uintptr_t)S & 15) == 0;
    if (fast) {
        for (int cb = warp; cb < nb / 16; cb += 8) {
            double v[16];
#pragma unroll
            for (int c = 0; c < 16; c++) v[c] = 0.0;
            for (int rb = 0; rb < nb / 64; rb++) {
                const int row = rb * 64 + 2 * lane;
                const double2 xr = *reinterpret_cast<const double2 *>(xp_s + row);
                double y0 = 0.0, y1 = 0.0;
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int col = cb * 16 + c;
                    double2 a = __ldg(reinterpret_cast<const double2 *>(S + (size_t)col * ld + row));
                    if (ABS) {
                        a.x = fabs(a.x);
                        a.y = fabs(a.y);
                    }
                    const double xc = xq_s[col];
                    y0 += a.x * xc;
                    y1 += a.y * xc;
                    v[c] += a.x * xr.x + a.y * xr.y;
                }
                ypart[warp][row] += y0;
                ypart[warp][row + 1] += y1;
            }
            double colsum = butterfly16(v, lane);
            const int col = cb * 16 + (lane & 15);
            if (lane < 16) yq_out[col] = colsum;
        }
    }
    // the general path: lanes walk rows one at a time; warps take 16-column
    // groups (16 accumulators and 16 loads in flight per lane keep the loop
    // in registers)
    const int nbr = (rows + 31) / 32, nbc = fast ? 0 : (cols + 15) / 16;
    for (int cb = warp; cb < nbc; cb += 8) {
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; c++) v[c] = 0.0;
        for (int rb = 0; rb < nbr; rb++) {
            const int row = rb * 32 + lane;
            const double xr = xp_s[row];
            double yrow = 0.0;
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const int col = cb * 16 + c;
                double a = (row < rows && col < cols)
                               ? S[(size_t)col * ld + row] : 0.0;
                if (ABS) a = fabs(a);
                // the part of a diagonal tile outside the stored triangle is
                // not referenced
                double a_dir = a, a_tr = a;
                if (diag) {
                    bool in = lower ? row >= col : row <= col;
                    a_dir = in ? a : 0.0;
                    a_tr = (in && row != col) ? a : 0.0;
                }
                yrow += a_dir * xq_s[col];
                v[c] += a_tr * xr;
            }
            ypart[warp][row] += yrow;
        }
        double colsum = butterfly16(v, lane);
        const int col = cb * 16 + (lane & 15);
        if (lane < 16) {
            if (diag) {
                if (col < cols) ypart[warp][col] += colsum;
            } else if (col < cols) {
                yq_out[col] = colsum;
            }
        }
    }
    __syncthreads();
    double *yp_out = part + ((size_t)p * mt + q) * nb;     // S x_q -> block p
    for (int i = tid; i < rows; i += SV_THREADS) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < 8; w++) s += ypart[w][i];
        yp_out[i] = s;
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v)
{
    atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// r_m = b_m - sum_q part[m][q] ; norms of x and r
__global__ void __launch_bounds__(SV_THREADS)
k_symv_reduce(plasma_desc_t A, const double *part, const double *b,
              const double *x, double *r, double *xnorm, double *rnorm,
              const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int m = blockIdx.x, mt = A.mt, nb = A.mb;
    const int rows = plasma_tile_mview(A, m);
    double xm = 0.0, rm = 0.0;
    for (int i = threadIdx.x; i < rows; i += SV_THREADS) {
        double s = 0.0;
        for (int q = 0; q < mt; q++) s += part[((size_t)m * mt + q) * nb + i];
        size_t gi = (size_t)m * nb + i;
        double v = (b ? b[gi] : 0.0) - s;
        if (r) r[gi] = b ? v : s;
        if (x) xm = fmax(xm, fabs(x[gi]));
        rm = fmax(rm, fabs(v));
    }
    for (int off = 16; off > 0; off >>= 1) {
        xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, off));
        rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, off));
    }
    if ((threadIdx.x & 31) == 0) {
        if (xnorm) atomic_max_nonneg(xnorm, xm);
        if (rnorm) atomic_max_nonneg(rnorm, rm);
    }
}

}  // namespace

extern "C" size_t plasma_cuda_symv_work(plasma_desc_t A)
{
    return (size_t)A.mt * A.mt * A.mb * sizeof(double);
}

// r = b - A x (b == NULL: r = A x).  x, b, r contiguous vectors of A.m
// entries, tile m at offset m*mb; xnorm/rnorm (device, may be NULL) receive
// max|x| and max|b - A x| (zeroed here).  work: plasma_cuda_symv_work bytes.
extern "C" int plasma_cuda_symv(cudaStream_t s, plasma_devstat_t *st,
                                plasma_enum_t uplo, plasma_desc_t A,
                                const double *x, const double *b, double *r,
                                double *xnorm, double *rnorm, double *work)
{
    if (A.precision != PlasmaRealDouble || A.mb != A.nb || A.mb > 512)
        return 0;
    if (xnorm) cudaMemsetAsync(xnorm, 0, sizeof(double), s);
    if (rnorm) cudaMemsetAsync(rnorm, 0, sizeof(double), s);
    if (A.mt == 0) return 1;
    const int mt = A.mt;
    const long long ntiles = (long long)mt * (mt + 1) / 2;
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    k_symv_tiles<false><<<(unsigned)ntiles, SV_THREADS, 0, s>>>(A, uplo, x, work, st);
    PLASMA_COUNT_LAUNCH();
    k_symv_reduce<<<mt, SV_THREADS, 0, s>>>(A, work, b, x, r, xnorm, rnorm, st);
    double n = A.m;
    plasma_prof_end(prof, s, PLASMA_KCLASS_AUX, 2.0 * n * n, 8.0 * n * (n + 1) / 2.0);
    return 1;
}

// ||A||_inf of symmetric A (uplo triangle) into *norm (device): the maximum
// row sum of |A| from one pass over the stored tiles.  work:
// plasma_cuda_symv_work bytes.  Returns 0 (nothing launched) when A is not
// an FP64 descriptor with square tiles of at most 512.
extern "C" int plasma_cuda_lansy_tiles(cudaStream_t s, plasma_devstat_t *st,
                                       plasma_enum_t uplo, plasma_desc_t A,
                                       double *norm, double *work)
{
    if (A.precision != PlasmaRealDouble || A.mb != A.nb || A.mb > 512)
        return 0;
    cudaMemsetAsync(norm, 0, sizeof(double), s);
    if (A.mt == 0) return 1;
    const int mt = A.mt;
    const long long ntiles = (long long)mt * (mt + 1) / 2;
    PLASMA_COUNT_LAUNCH();
    int prof = plasma_prof_begin(s);
    k_symv_tiles<true><<<(unsigned)ntiles, SV_THREADS, 0, s>>>(A, uplo, nullptr, work, st);
    PLASMA_COUNT_LAUNCH();
    k_symv_reduce<<<mt, SV_THREADS, 0, s>>>(A, work, nullptr, nullptr, nullptr, nullptr,
                                            norm, st);
    double n = A.m;
    plasma_prof_end(prof, s, PLASMA_KCLASS_AUX, n * n, 8.0 * n * (n + 1) / 2.0);
    return 1;
}
