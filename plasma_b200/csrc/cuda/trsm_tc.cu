// trsm_tc.cu -- the panel triangular solve of the FP32 Cholesky on the
// fifth-generation tensor cores (tcgen05), for the tile columns below a
// diagonal tile:
//
//     X L_kk^T = A(m,k),   m = mlo .. mhi-1
//
// (compute/pzpotrf.c:47-56, plasma_core_strsm Right, Lower, Trans, NonUnit
// on every tile under the diagonal one).  The nb columns of L_kk are taken in
// 64-column blocks; block j of X solves
//
//     X_j L_jj^T = Y_j,   Y_j = A_j - sum_{i<j} X_i L_ji^T
//
// as one product X_j = Y_j (L_jj^-1)^T, with the inverse of the 64 x 64
// diagonal block formed in FP64 once per step (k_trsm_prep).  So every part
// of the solve is a tensor-core product and no thread walks a substitution
// chain.  k_trsm_prep writes one operand image of L_kk, W, column-major
// nb x nb: the diagonal 64-blocks replaced by their inverses (zero above
// their diagonal), the blocks below kept, both rounded to TF32 and split
// w = hi + lo (hi = tf32(w), lo = tf32(w - hi)) when the factor is FP32.
//
// k_trsm_tc: one CTA per 128 rows of one tile.
//   warp 4  : TMA producer -- per block j the diagonal block W(j,j) (two
//             buffers) and the blocks below it, W(j+1 .., j), as one operand
//             of N = 64 (nblk-1-j) (one buffer);
//   warp 5  : tensor-memory allocation and the MMA issuer (one thread);
//   warps 0-3: rows 32w .. 32w+31 -- per block j: read the accumulator of
//             block j (tcgen05.ld), Y_j = A_j - acc, split Y_j and write it to
//             tensor memory (tcgen05.st) as the A operand of X_j = Y_j W_jj;
//             read X_j back and write its split to tensor memory as the A
//             operand of the update of every block to its right (one MMA
//             chain of N up to 192 into their adjacent accumulators);
//   warps 6-9: the same rows (tensor lanes 32 (w mod 4) ..) -- read X_j,
//             stage it, and its rounded copies when the trailing update takes
//             TF32 operands, in shared memory for TMA stores to A(m,k) and to
//             the panel buffer the update reads; the stores stay off the
//             chain of dependent steps above (the X product of block j+1
//             only waits until these warps have read X_j).
#include "common.cuh"
#include "tc.cuh"
#include "inv64.cuh"

namespace {

constexpr int TS_M = 128;              // rows per CTA (MMA M, tensor lanes)
constexpr int TS_B = 64;               // column block (MMA K; N of the X product)
constexpr int TS_THREADS = 320;
constexpr int TS_STORE_WARP0 = 6;
constexpr int TS_PRODUCER_WARP = 4;
constexpr int TS_MMA_WARP = 5;
constexpr int TS_PART_BYTES = TS_B * TS_B * 4;           // one 64 x 64 block
constexpr int TS_MAXU = 3;                               // blocks below the diagonal one
constexpr int TS_WX = 0;                                 // two buffers of W(j,j), hi and lo
constexpr int TS_WU = TS_WX + 2 * 2 * TS_PART_BYTES;     // W(j+1.., j): hi, then lo
constexpr int TS_STG = TS_WU + 2 * TS_MAXU * TS_PART_BYTES;
constexpr int TS_STG_WARP = 3 * 32 * 32 * 4;             // X, hi, lo: 32 x 32 each
constexpr int TS_SMEM = TS_STG + 4 * TS_STG_WARP + 1024;
constexpr uint32_t TS_CHUNK = TS_B * 128;                // one MN chunk: 64 K-rows
constexpr uint32_t TS_SBO = 512;                         // 4 K-rows per atom
constexpr int TS_PREP_SMEM = (2 * TS_B * (TS_B + 1) + TS_B * (TS_B / 2 + 1)) * 8;

struct TsArgs {
    plasma_desc_t A;
    int k, mlo;
    int split;          // 3: hi/lo products (FP32 factor), 1: one TF32 product
    int panel;          // write the rounded copies of the solved tiles
    int poff;           // panel tile of row tile m: poff + m (hi), + pstride (lo)
    int pstride;
};

__device__ __forceinline__ uint32_t tf32_round(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
        :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]),
           "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]),
           "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
           "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
           "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]),
           "r"(r[31])
        : "memory");
}

// D (tensor memory) (+)= A (tensor memory, M x K) * B (shared memory)
__device__ __forceinline__ void mma_ta(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
        :: "r"(d), "r"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit1(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

// F32 accumulator, TF32 A and B, A K-major (tensor memory), B MN-major,
// M = 128, N = n
__device__ __forceinline__ uint32_t ts_idesc(int n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TS_M >> 4) << 24);
}

// tile (r, c) .. (r+31, c+31) of the 3-D tile map <- 32 x 32 block staged
// column-major in shared memory
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0,
                                             int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
        :: "l"(map), "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2) : "memory");
}

// The split of one thread's 32 values: hi = tf32(v), lo = tf32(v - hi).
__device__ __forceinline__ void split32(const float (&v)[32], uint32_t (&hi)[32],
                                        uint32_t (&lo)[32], int split)
{
#pragma unroll
    for (int i = 0; i < 32; i++) {
        hi[i] = tf32_round(v[i]);
        lo[i] = split == 3 ? tf32_round(v[i] - __uint_as_float(hi[i])) : 0u;
    }
}

__global__ void __launch_bounds__(TS_THREADS, 1)
k_trsm_tc(const __grid_constant__ CUtensorMap wmap, const __grid_constant__ CUtensorMap amap,
          const __grid_constant__ CUtensorMap pmap, TsArgs g, plasma_devstat_t *st)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t fullx_bar[2], emptyx_bar[2], fullu_bar, emptyu_bar;
    __shared__ uint64_t y_bar, x_bar, xr_bar, acc_bar, xs_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    __shared__ int failed_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = g.mlo + blockIdx.x;
    const int rows = plasma_tile_mview(g.A, m);
    const int r0 = blockIdx.y * TS_M;
    if (tid == 0) failed_s = plasma_failed(st) ? 1 : 0;
    __syncthreads();
    if (failed_s || r0 >= rows) return;

    const int nb = g.A.mb;
    const int nblk = nb / TS_B;
    const int parts = g.split == 3 ? 2 : 1;
    // tensor memory: acc_j (j = 1 .. nblk-1) at 64 (j-1), then X, A hi, A lo
    const uint32_t c_x = (uint32_t)(nblk - 1) * TS_B;
    const uint32_t c_ahi = c_x + TS_B, c_alo = c_ahi + TS_B;
    const uint32_t tmem_cols = nb == 256 ? 512u : 256u;   // 384 or 256 used
    unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);

    if (tid == 0) {
        for (int s = 0; s < 2; s++) {
            mbar_init(&fullx_bar[s], 1);
            mbar_init(&emptyx_bar[s], 1);
        }
        mbar_init(&fullu_bar, 1);
        mbar_init(&emptyu_bar, 1);
        mbar_init(&y_bar, 4);
        mbar_init(&xr_bar, 4);
        mbar_init(&x_bar, 1);
        mbar_init(&acc_bar, 1);
        mbar_init(&xs_bar, 4);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == TS_MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base_s)), "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    if (warp == TS_PRODUCER_WARP && lane == 0) {
        // ---------------- producer: W(j,j), then W(j+1 .., j), j = 0 ..
        for (int j = 0; j < nblk; j++) {
            unsigned char *wx = sm + TS_WX + (j & 1) * 2 * TS_PART_BYTES;
            if (j >= 2 && !mbar_wait(&emptyx_bar[j & 1], ((j >> 1) - 1) & 1, &abort_s)) break;
            mbar_expect_tx(&fullx_bar[j & 1], (uint32_t)(parts * TS_PART_BYTES));
            for (int p = 0; p < parts; p++)
                tma_load_4d(wx + p * TS_PART_BYTES, &wmap, &fullx_bar[j & 1], 0, TS_B * j,
                            (TS_B / 32) * j, p);
            const int r = nblk - 1 - j;
            if (r == 0) break;
            if (j >= 1 && !mbar_wait(&emptyu_bar, (j - 1) & 1, &abort_s)) break;
            mbar_expect_tx(&fullu_bar, (uint32_t)(parts * r * TS_PART_BYTES));
            for (int p = 0; p < parts; p++)
                for (int t = 0; t < r; t++)
                    tma_load_4d(sm + TS_WU + (p * TS_MAXU + t) * TS_PART_BYTES, &wmap,
                                &fullu_bar, 0, TS_B * j, (TS_B / 32) * (j + 1 + t), p);
        }
    } else if (warp == TS_MMA_WARP && lane == 0) {
        // ---------------- MMA issuer
        // D (+)= A (tensor memory, hi/lo at c_ahi/c_alo) x B (N x 64, hi then lo
        // at `bl` bytes further)
        auto products = [&](uint32_t d, const unsigned char *b, int bl, int n, uint32_t first) {
            const uint32_t idesc = ts_idesc(n);
#pragma unroll
            for (int kk = 0; kk < TS_B / 8; kk++) {
                const uint64_t bh = smem_desc(b + kk * 8 * 128, TS_CHUNK, TS_SBO, 1u);
                const uint32_t ah = tmem + c_ahi + 8 * kk;
                const uint32_t acc = (kk > 0 || first) ? 1u : 0u;
                if (parts == 2) {
                    const uint64_t blo = smem_desc(b + bl + kk * 8 * 128, TS_CHUNK, TS_SBO, 1u);
                    const uint32_t al = tmem + c_alo + 8 * kk;
                    mma_ta(tmem + d, al, bh, idesc, acc);         // small terms first
                    mma_ta(tmem + d, ah, blo, idesc, 1u);
                    mma_ta(tmem + d, ah, bh, idesc, 1u);
                } else {
                    mma_ta(tmem + d, ah, bh, idesc, acc);
                }
            }
        };
        for (int j = 0; j < nblk; j++) {
            if (!mbar_wait(&y_bar, j & 1, &abort_s)) break;
            if (!mbar_wait(&fullx_bar[j & 1], (j >> 1) & 1, &abort_s)) break;
            // X_{j-1} has been read by the store warps
            if (j > 0 && !mbar_wait(&xs_bar, (j - 1) & 1, &abort_s)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            products(c_x, sm + TS_WX + (j & 1) * 2 * TS_PART_BYTES, TS_PART_BYTES, TS_B, 0u);
            mma_commit1(&emptyx_bar[j & 1]);
            mma_commit1(&x_bar);
            const int r = nblk - 1 - j;
            if (r == 0) break;
            if (!mbar_wait(&xr_bar, j & 1, &abort_s)) break;
            if (!mbar_wait(&fullu_bar, j & 1, &abort_s)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            products((uint32_t)j * TS_B, sm + TS_WU, TS_MAXU * TS_PART_BYTES, TS_B * r,
                     j > 0 ? 1u : 0u);
            mma_commit1(&emptyu_bar);
            mma_commit1(&acc_bar);
        }
    } else if (warp < 4) {
        // ---------------- rows 32w .. 32w+31 of this CTA: the solve
        const int row = r0 + 32 * warp + lane;
        const bool live = row < rows;
        const float *Bt = (const float *)plasma_tile_addr(g.A, m, g.k);
        const int ldb = plasma_tile_mmain(g.A, m);
        const uint32_t lanes = (uint32_t)(32 * warp) << 16;
        float b[TS_B];          // the right-hand side of block j
#pragma unroll
        for (int c = 0; c < TS_B; c++) b[c] = live ? Bt[(size_t)c * ldb + row] : 0.f;
        for (int j = 0; j < nblk; j++) {
            // Y_j = A_j - acc_j: the updates by blocks < j are complete (and
            // the A operand they read is free) once acc_bar fires for j - 1
            if (j > 0) {
                const bool ok = __all_sync(0xffffffffu,
                                           mbar_wait(&acc_bar, (j - 1) & 1, &abort_s));
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float v[32];
                if (j > 0) {
                    tmem_ld32(tmem + lanes + (uint32_t)(j - 1) * TS_B + 32 * h, v);
#pragma unroll
                    for (int i = 0; i < 32; i++) v[i] = b[32 * h + i] - v[i];
                } else {
#pragma unroll
                    for (int i = 0; i < 32; i++) v[i] = b[32 * h + i];
                }
                uint32_t hi[32], lo[32];
                split32(v, hi, lo, g.split);
                tmem_st32(tmem + lanes + c_ahi + 32 * h, hi);
                if (g.split == 3) tmem_st32(tmem + lanes + c_alo + 32 * h, lo);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&y_bar);
            if (j + 1 == nblk) break;
            // the next block's right-hand side while the product runs
#pragma unroll
            for (int c = 0; c < TS_B; c++)
                b[c] = live ? Bt[(size_t)(TS_B * (j + 1) + c) * ldb + row] : 0.f;
            const bool okx = __all_sync(0xffffffffu, mbar_wait(&x_bar, j & 1, &abort_s));
            if (!okx) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float v[32];
                tmem_ld32(tmem + lanes + c_x + 32 * h, v);
                uint32_t hi[32], lo[32];
                split32(v, hi, lo, g.split);
                tmem_st32(tmem + lanes + c_ahi + 32 * h, hi);
                if (g.split == 3) tmem_st32(tmem + lanes + c_alo + 32 * h, lo);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&xr_bar);
        }
    } else if (warp >= TS_STORE_WARP0) {
        // ---------------- the same rows: X_j to A(m,k) and the panel copies
        const int q = warp & 3;
        const uint32_t lanes = (uint32_t)(32 * q) << 16;
        const float *Bt = (const float *)plasma_tile_addr(g.A, m, g.k);
        const int atile = (int)(((const char *)Bt - (const char *)g.A.matrix) /
                                ((size_t)nb * nb * 4));
        float *stg = (float *)(sm + TS_STG + q * TS_STG_WARP);
        bool staged = false;    // a store group of this warp may still read stg
        for (int j = 0; j < nblk; j++) {
            const bool okx = __all_sync(0xffffffffu, mbar_wait(&x_bar, j & 1, &abort_s));
            if (!okx) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float x[TS_B];
            tmem_ld32(tmem + lanes + c_x, *reinterpret_cast<float (*)[32]>(&x[0]));
            tmem_ld32(tmem + lanes + c_x + 32, *reinterpret_cast<float (*)[32]>(&x[32]));
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&xs_bar);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                // the previous group of this warp must be done reading stg
                if (staged && lane == 0) bulk_wait_read<0>();
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 32; i++) {
                    const float v = x[32 * h + i];
                    const uint32_t hi = tf32_round(v);
                    stg[i * 32 + lane] = v;
                    stg[1024 + i * 32 + lane] = __uint_as_float(hi);
                    stg[2048 + i * 32 + lane] =
                        __uint_as_float(tf32_round(v - __uint_as_float(hi)));
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    const int rr = r0 + 32 * q, cc = TS_B * j + 32 * h;
                    tma_store_3d(&amap, stg, rr, cc, atile);
                    if (g.panel) {
                        tma_store_3d(&pmap, stg + 1024, rr, cc, g.poff + m);
                        if (g.split == 3)
                            tma_store_3d(&pmap, stg + 2048, rr, cc, g.poff + g.pstride + m);
                    }
                    bulk_commit();
                }
                staged = true;
            }
        }
        if (lane == 0) bulk_wait_all();
        __syncwarp();
    }
    // ---------------- teardown
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_s) {
        if (tid == 0) {
            plasma_fail(st, PlasmaErrorInternal, 0);
            // a bounded time for issued MMAs and copies to land before
            // tensor and shared memory are released
            long long t0 = clock64();
            while (clock64() - t0 < 200000000LL) {}
        }
        __syncthreads();
    }
    if (warp == TS_MMA_WARP) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(tmem_cols));
    }
}

// ---------------------------------------------------------------------------
// W: the operand image of L_kk.  CTA j < nblk inverts the diagonal block
// L_jj in FP64 -- the eight 8 x 8 blocks by substitution (a thread per
// column), then [A 0; B C]^-1 = [A^-1 0; -C^-1 B A^-1  C^-1] at sizes 16, 32
// and 64 (the products of the last two on DMMA) -- and writes it, zero above the diagonal; each further CTA copies one
// of the 64 x 64 blocks below the diagonal ones.  Both are rounded and split
// as the products read them.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void put_w(float *__restrict__ whi, float *__restrict__ wlo,
                                      size_t e, float v, int split)
{
    const uint32_t hi = tf32_round(v);
    whi[e] = __uint_as_float(hi);
    if (split == 3) wlo[e] = __uint_as_float(tf32_round(v - __uint_as_float(hi)));
}

__global__ void __launch_bounds__(256)
k_trsm_prep(plasma_desc_t A, int k, float *w, int split, const plasma_devstat_t *st)
{
    extern __shared__ double prep_smem[];
    constexpr int LD = TS_B + 1, TLD = TS_B / 2 + 1;
    double (*Ls)[LD] = reinterpret_cast<double (*)[LD]>(prep_smem);
    double (*Iv)[LD] = Ls + TS_B;
    double (*Tm)[TLD] = reinterpret_cast<double (*)[TLD]>(Iv + TS_B);
    const int tid = threadIdx.x;
    const int nb = A.mb, nblk = nb / TS_B;
    const float *__restrict__ L = (const float *)plasma_tile_addr(A, k, k);
    const int ldl = plasma_tile_mmain(A, k);
    float *whi = w, *wlo = w + (size_t)nb * nb;
    constexpr int PER = TS_B * TS_B / 256;     // elements of a block per thread

    if ((int)blockIdx.x >= nblk) {
        // the block (j2, j), j2 > j, numbered column by column
        int b = blockIdx.x - nblk, j = 0;
        while (b >= nblk - 1 - j) { b -= nblk - 1 - j; j++; }
        const int r0 = TS_B * (j + 1 + b), c0 = TS_B * j;
        float v[PER];
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + 256 * q;
            v[q] = L[(size_t)(c0 + e / TS_B) * ldl + r0 + e % TS_B];
        }
        if (plasma_failed(st)) return;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + 256 * q;
            put_w(whi, wlo, (size_t)(c0 + e / TS_B) * nb + r0 + e % TS_B, v[q], split);
        }
        return;
    }

    const int base = TS_B * blockIdx.x;
    {
        float v[PER];
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + 256 * q;
            v[q] = L[(size_t)(base + e / TS_B) * ldl + base + e % TS_B];
        }
        if (plasma_failed(st)) return;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + 256 * q, i = e % TS_B, c = e / TS_B;
            Ls[i][c] = i >= c ? (double)v[q] : 0.0;
            Iv[i][c] = 0.0;
        }
    }
    __syncthreads();
    inv_lower64(Ls, Iv, Tm, false);
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int e = tid + 256 * q, i = e % TS_B, c = e / TS_B;
        put_w(whi, wlo, (size_t)(base + c) * nb + base + i, i >= c ? (float)Iv[i][c] : 0.f,
              split);
    }
}

// W map: 4-D over the column-major nb x nb image parts, as the trailing
// update's operand map -- dim 0: 32 rows (128 bytes), dim 1: columns (K),
// dim 2: 32-row chunks, dim 3: part (hi, lo) -- with a box of one 64 x 64
// block: {32, 64, 2, 1}.
bool encode_w_map(CUtensorMap *map, void *base, int nb, int parts)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr) return false;
    cuuint64_t dims[4] = {32, (cuuint64_t)nb, (cuuint64_t)(nb / 32), (cuuint64_t)parts};
    cuuint64_t strides[3] = {(cuuint64_t)nb * 4, 128, (cuuint64_t)nb * nb * 4};
    cuuint32_t box[4] = {32, (cuuint32_t)TS_B, (cuuint32_t)(TS_B / 32), 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 3-D map over column-major nb x nb tiles {rows, columns, tile}, box 32 x 32
bool encode_tiles_32(CUtensorMap *map, void *base, int nb, long long ntiles)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr || ntiles <= 0) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nb, (cuuint64_t)nb, (cuuint64_t)ntiles};
    cuuint64_t strides[2] = {(cuuint64_t)nb * 4, (cuuint64_t)nb * nb * 4};
    cuuint32_t box[3] = {32, 32, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

extern "C" void plasma_cuda_panel_layout(plasma_desc_t A, int k, int full, int *poff,
                                         int *pstride);

// Bytes of the W image (both parts) for tiles of nb.
extern "C" size_t plasma_cuda_trsm_tc_bytes(int nb)
{
    return 2 * (size_t)nb * nb * sizeof(float);
}

// The panel solve of step k on the tensor cores.  `wimg`: 1024-byte aligned
// scratch of plasma_cuda_trsm_tc_bytes(nb).  `panel` (may be null): the
// rounded operand copies of the trailing update for `mode` in the layout
// `full` (plasma_cuda_panel_round's); written here when the update takes
// TF32 operands.  Returns 0 when not eligible (nothing launched), 1 when the
// solve ran, 2 when it also wrote the panel copies.
extern "C" int plasma_cuda_trsm_tc(cudaStream_t s, plasma_devstat_t *st, int mode,
                                   plasma_desc_t A, int k, int mlo, int mhi, void *wimg,
                                   void *panel, int full)
{
    if (!plasma_cuda_update_tc_ok(A, PlasmaLower) || wimg == nullptr ||
        ((uintptr_t)wimg & 1023) != 0 || plasma_tile_mview(A, k) != A.nb)
        return 0;
    static int env = -1;
    if (env < 0) {
        // PLASMA_TRSM_TC=0 keeps the panel solve on the mma.sync kernel
        const char *e = getenv("PLASMA_TRSM_TC");
        env = e ? atoi(e) != 0 : 1;
    }
    if (!env) return 0;
    if (mhi <= mlo) return 1;
    const int nb = A.mb;
    const int split = mode == PLASMA_TC_TF32 || mode == PLASMA_TC_BF16 ? 1 : 3;
    const int parts = split == 3 ? 2 : 1;
    int poff = 0, pstride = 0;
    const bool write_panel = panel != nullptr &&
                             (mode == PLASMA_TC_TF32X3 || mode == PLASMA_TC_TF32);
    if (write_panel) plasma_cuda_panel_layout(A, k, full, &poff, &pstride);
    const long long atiles = (long long)(plasma_desc_storage_bytes(A) / ((size_t)nb * nb * 4));
    CUtensorMap wmap, amap, pmap;
    if (!encode_w_map(&wmap, wimg, nb, parts) ||
        !encode_tiles_32(&amap, A.matrix, nb, atiles) ||
        !encode_tiles_32(&pmap, write_panel ? panel : A.matrix, nb,
                         write_panel ? (long long)parts * pstride : atiles))
        return 0;

    TsArgs g;
    g.A = A;
    g.k = k;
    g.mlo = mlo;
    g.split = split;
    g.panel = write_panel ? 1 : 0;
    g.poff = poff;
    g.pstride = pstride;

    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_trsm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TS_SMEM);
        cudaFuncSetAttribute(k_trsm_prep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TS_PREP_SMEM);
    }
    double rows = 0;
    for (int m = mlo; m < mhi; m++) rows += plasma_tile_mview(A, m);
    int prof = plasma_prof_begin(s);
    PLASMA_COUNT_LAUNCH();
    const int nblk = nb / TS_B;
    k_trsm_prep<<<nblk + nblk * (nblk - 1) / 2, 256, TS_PREP_SMEM, s>>>(A, k, (float *)wimg, split, st);
    PLASMA_COUNT_LAUNCH();
    dim3 grid((unsigned)(mhi - mlo), (unsigned)(nb / TS_M));
    static int paired = -1;
    if (paired < 0) {
        const char *e = getenv("PLASMA_TRSM_PAIRED");
        paired = e ? atoi(e) != 0 : 1;
    }
    if (paired && grid.y == 2) {
        // the two halves of a tile as a cluster of two CTAs: they are
        // scheduled on a pair of SMs at once, like the trailing update's
        // CTA pairs, so the solve and the update hand SMs to each other in
        // pairs (the CTAs share nothing)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(TS_THREADS);
        cfg.dynamicSmemBytes = TS_SMEM;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 1;
        at[0].val.clusterDim.y = 2;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_trsm_tc, wmap, amap, pmap, g, st);
    } else {
        k_trsm_tc<<<grid, TS_THREADS, TS_SMEM, s>>>(wmap, amap, pmap, g, st);
    }
    plasma_prof_end(prof, s, PLASMA_KCLASS_TRSM, rows * nb * nb, 2.0 * rows * nb * 4.0);
    return write_panel ? 2 : 1;
}
