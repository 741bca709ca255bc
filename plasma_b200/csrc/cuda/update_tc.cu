// update_tc.cu -- trailing update of the FP32 Cholesky on the fifth-
// generation tensor cores (tcgen05, accumulators in tensor memory).
//
//     C(m,n) -= A(m,k) * A(n,k)^T     C in FP32
//
// This is the SYRK/GEMM part of plasma_pspotrf (the FP32 tile Cholesky that
// the reference runs inside dsposv, compute/zcposv.c:452 ->
// compute/pzpotrf.c:57-77).  Three product precisions, all accumulated in
// FP32 in tensor memory:
//   TF32   : one kind::tf32 MMA per k-step on the TF32-rounded panel;
//   BF16   : one kind::f16 MMA per k-step on the BF16-rounded panel;
//   TF32X3 : the panel split as a = hi + lo (hi = tf32(a), lo = tf32(a - hi))
//            and a*b formed as lo*hi + hi*lo + hi*hi, three kind::tf32 MMAs,
//            which keeps about 22 bits of every product (the FP32 factor);
//   BF16X6 : the panel split in three BF16 parts, a = h + m + l (h = bf16(a),
//            m = bf16(a - h), l = bf16(a - h - m)), and a*b formed from the six
//            products whose order is at most 2^-16 (l*h, h*l, m*m, m*h, h*m,
//            h*h), six kind::f16 MMAs: about 23 bits of every product, the
//            same tensor time as TF32X3 (a BF16 MMA covers twice the K) and
//            6 instead of 8 operand bytes per element (the FP32 factor on
//            256-wide tiles, CTA-pair kernel only).
//
// One CTA owns a run of `ipc` consecutive work items (a 128 x nb block of one
// output tile each; items of one tile column are adjacent, so they share the
// B operand in L2):
//   warp 0     : TMA producer -- 4-D tensor maps over the column-major panel
//                tiles (128-byte swizzle; 32-byte swizzle atoms for TF32, the
//                only MN-major TF32 layout), a ring of 48 KB stages (4 for
//                TF32X3, 3 otherwise);
//   warp 1     : MMA issuer -- one thread issues tcgen05.mma (M = 128, N = nb,
//                MN-major A and B), tcgen05.commit frees a stage and, after
//                the last k-step of an item, publishes its accumulator;
//   warp 2     : tensor-memory allocation (two accumulators of nb columns);
//   warps 4-11 : epilogue -- tcgen05.ld of an accumulator, -P staged in
//                shared memory in 32 x 32 blocks (zero above the diagonal of
//                diagonal tiles) and added to C by TMA reductions
//                (cp.reduce.async.bulk.tensor .add.f32): the read-modify-write
//                of C runs in the memory system, asynchronously, one add per
//                element, so the result is deterministic; then the
//                accumulator is handed back to the MMA warp.
// With two accumulators the epilogue of item j overlaps the MMAs of item j+1.
// CTAs stay short (a few items) so that the kernels of the critical panel
// stream find free SMs while a large update runs.  Every mbarrier wait is
// bounded (about 2 s); on expiry the CTA records PlasmaErrorInternal, lets
// what it issued drain and frees its tensor memory.
#include "common.cuh"
#include "tc.cuh"

#include <cuda_bf16.h>
#include <stdlib.h>

namespace {

constexpr int TC_M = 128;
constexpr int TC_THREADS = 384;          // 12 warps
constexpr int TC_EPI_WARP0 = 4;
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_STAGE_BYTES = 48 * 1024;
constexpr int TC_EPI_BUF_BYTES = 32 * 32 * 4;

enum { MODE_TF32 = PLASMA_TC_TF32, MODE_BF16 = PLASMA_TC_BF16,
       MODE_TF32X3 = PLASMA_TC_TF32X3, MODE_BF16X6 = PLASMA_TC_BF16X6 };

template <int MODE>
struct Geo {
    static constexpr bool HALF16 = MODE == MODE_BF16 || MODE == MODE_BF16X6;
    static constexpr int ESZ = HALF16 ? 2 : 4;
    static constexpr int MNBOX = 128 / ESZ;           // elements per 128-byte row
    static constexpr int BK = MODE == MODE_BF16 ? 64
                            : (MODE == MODE_TF32 || MODE == MODE_BF16X6) ? 32 : 16;
    static constexpr int KI = HALF16 ? 16 : 8;        // K per instruction
    static constexpr int PARTS = MODE == MODE_TF32X3 ? 2 : MODE == MODE_BF16X6 ? 3 : 1;
    static constexpr uint32_t LAYOUT = HALF16 ? 2u : 1u;
    static constexpr uint32_t SBO = HALF16 ? 1024u : 512u;
    static constexpr int CHUNK = BK * 128;            // one MN chunk of a stage
    static constexpr int A_BYTES = (TC_M / MNBOX) * CHUNK;
    // TF32X3 moves twice the operand bytes per product: a deeper ring (more
    // bytes in flight against the L2 latency), one epilogue buffer per warp
    static constexpr int STAGES = MODE == MODE_TF32X3 ? 4 : 3;
    static constexpr int EPI_BUFS = MODE == MODE_TF32X3 ? 1 : 2;
    static constexpr int SMEM = STAGES * TC_STAGE_BYTES +
                                TC_EPI_WARPS * EPI_BUFS * TC_EPI_BUF_BYTES + 1024;
};

__device__ __forceinline__ uint32_t instr_desc(int mode, int n)
{
    uint32_t fmt = mode == MODE_BF16 ? 1u : 2u;   // BF16 : TF32
    return (1u << 4)                 // D format F32
         | (fmt << 7) | (fmt << 10)  // A, B format
         | (1u << 15) | (1u << 16)   // A, B MN-major
         | ((uint32_t)(n >> 3) << 17)
         | ((uint32_t)(TC_M >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b,
                                    uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;      // no output lane disabled
    if (MODE != MODE_BF16)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
            :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
            :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}

struct TcArgs {
    plasma_desc_t A;    // FP32 general or packed-lower descriptor holding C
    int k, nlo, nhi;
    int poff;           // operand tile of panel row m: poff + m (first part)
    int mt;             // tiles per part in the operand map (part p at +p*mt)
    long long nitems;
    int ipc;            // items per CTA
};

// work item -> (m, n, si); items run over si fastest, then m, then n
__device__ __forceinline__ void tc_item(const TcArgs &g, long long w, int &m, int &n,
                                        int &si)
{
    const int sb = g.A.mb / TC_M;
    long long p = w / sb;
    si = (int)(w - p * sb);
    n = g.nlo;
    while (n < g.nhi - 1 && p >= g.A.mt - n) { p -= g.A.mt - n; n++; }
    m = n + (int)p;
}

template <int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1)
k_update_tc(const __grid_constant__ CUtensorMap opmap,
            const __grid_constant__ CUtensorMap cmap, TcArgs g,
            plasma_devstat_t *st)
{
    using G = Geo<MODE>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int TC_STAGES = G::STAGES;
    constexpr int TC_EPI_BUFS = G::EPI_BUFS;
    __shared__ uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES];
    __shared__ uint64_t tfull_bar[2], tempty_bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    if (plasma_failed(st)) return;
    const long long first = (long long)blockIdx.x * g.ipc;
    if (first >= g.nitems) return;
    const int nit = (int)min((long long)g.ipc, g.nitems - first);

    const int nb = g.A.mb;                         // N of the MMA
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *stage_base =
        (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int b_bytes = (nb / G::MNBOX) * G::CHUNK;
    const int stage_bytes = G::PARTS * (G::A_BYTES + b_bytes);
    const int nkb = nb / G::BK;                    // K = nb
    const uint32_t tmem_cols = 2 * nb;

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull_bar[a], 1);
            mbar_init(&tempty_bar[a], TC_EPI_WARPS);
        }
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base_s)), "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    if (warp == 0 && lane == 0) {
        // ---------------- producer
        int it = 0;                                   // k-blocks issued so far
        bool ok = true;
        for (int j = 0; j < nit && ok; j++) {
            int m, n, si;
            tc_item(g, first + j, m, n, si);
            const int i0 = si * TC_M;
            for (int kb = 0; kb < nkb; kb++, it++) {
                const int s = it % TC_STAGES;
                if (it >= TC_STAGES &&
                    !mbar_wait(&empty_bar[s], ((it / TC_STAGES) - 1) & 1, &abort_s)) {
                    ok = false;
                    break;
                }
                unsigned char *sp = stage_base + s * TC_STAGE_BYTES;
                mbar_expect_tx(&full_bar[s], (uint32_t)stage_bytes);
#pragma unroll
                for (int p = 0; p < G::PARTS; p++) {
                    unsigned char *sa = sp + p * G::A_BYTES;
                    unsigned char *sb = sp + G::PARTS * G::A_BYTES + p * b_bytes;
                    const int toff = g.poff + p * g.mt;
                    tma_load_4d(sa, &opmap, &full_bar[s], 0, kb * G::BK,
                                i0 / G::MNBOX, m + toff);
                    for (int c = 0; c < nb / TC_M; c++)
                        tma_load_4d(sb + c * G::A_BYTES, &opmap, &full_bar[s], 0,
                                    kb * G::BK, c * (TC_M / G::MNBOX), n + toff);
                }
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = instr_desc(MODE, nb);
        int it = 0;
        bool ok = true;
        for (int j = 0; j < nit && ok; j++) {
            const int a = j & 1;
            if (j >= 2 && !mbar_wait(&tempty_bar[a], ((j >> 1) - 1) & 1, &abort_s))
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc_t = tmem + (uint32_t)(a * nb);
            for (int kb = 0; kb < nkb; kb++, it++) {
                const int s = it % TC_STAGES;
                if (!mbar_wait(&full_bar[s], (it / TC_STAGES) & 1, &abort_s)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                unsigned char *sp = stage_base + s * TC_STAGE_BYTES;
                unsigned char *sa_hi = sp;
                unsigned char *sb_hi = sp + G::PARTS * G::A_BYTES;
#pragma unroll
                for (int kk = 0; kk < G::BK / G::KI; kk++) {
                    const uint32_t acc_on = (kb | kk) != 0;
                    uint64_t da = smem_desc(sa_hi + kk * G::KI * 128, G::CHUNK, G::SBO,
                                            G::LAYOUT);
                    uint64_t db = smem_desc(sb_hi + kk * G::KI * 128, G::CHUNK, G::SBO,
                                            G::LAYOUT);
                    if (MODE == MODE_TF32X3) {
                        unsigned char *sa_lo = sp + G::A_BYTES;
                        unsigned char *sb_lo = sb_hi + b_bytes;
                        uint64_t dal = smem_desc(sa_lo + kk * G::KI * 128, G::CHUNK, G::SBO,
                                                 G::LAYOUT);
                        uint64_t dbl = smem_desc(sb_lo + kk * G::KI * 128, G::CHUNK, G::SBO,
                                                 G::LAYOUT);
                        // small terms first
                        mma<MODE>(acc_t, dal, db, idesc, acc_on);
                        mma<MODE>(acc_t, da, dbl, idesc, 1u);
                        mma<MODE>(acc_t, da, db, idesc, 1u);
                    } else {
                        mma<MODE>(acc_t, da, db, idesc, acc_on);
                    }
                }
                mma_commit(&empty_bar[s]);
            }
            if (ok) mma_commit(&tfull_bar[a]);
        }
    } else if (warp >= TC_EPI_WARP0) {
        // ---------------- epilogue: warp -> TMEM lane quarter and column half
        const int e = warp - TC_EPI_WARP0;
        const int q = warp & 3;                  // lanes 32q .. 32q+31
        const int half = e / 4;                  // columns [half*nb/2, ...)
        float *stage_epi = (float *)(stage_base + TC_STAGES * TC_STAGE_BYTES) +
                           (size_t)e * TC_EPI_BUFS * (TC_EPI_BUF_BYTES / 4);
        int nchunk = 0;
        for (int j = 0; j < nit; j++) {
            const int a = j & 1;
            const bool ok = __all_sync(0xffffffffu,
                                       mbar_wait(&tfull_bar[a], (j >> 1) & 1, &abort_s));
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int m, n, si;
            tc_item(g, first + j, m, n, si);
            const int tile = (int)(((const char *)plasma_tile_addr(g.A, m, n) -
                                    (const char *)g.A.matrix) / ((size_t)nb * nb * 4));
            const int r0 = si * TC_M + 32 * q;   // first row of this warp
            const int row = r0 + lane;
            const bool diag = m == n;
            const int c0 = half * (nb / 2);
            for (int cc = c0; cc < c0 + nb / 2; cc += 32, nchunk++) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * nb + cc), v);
                float *buf = stage_epi + (nchunk % TC_EPI_BUFS) * (TC_EPI_BUF_BYTES / 4);
                // the reduction that last read this buffer must be done with it
                if (nchunk >= TC_EPI_BUFS && lane == 0) bulk_wait_read<TC_EPI_BUFS - 1>();
                __syncwarp();
#pragma unroll
                for (int jj = 0; jj < 32; jj++) {
                    const int col = cc + jj;
                    buf[jj * 32 + lane] = (!diag || row >= col) ? -v[jj] : 0.f;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    tma_reduce_add_3d(&cmap, buf, r0, cc, tile);
                    bulk_commit();
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[a]);
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
            // Give the MMAs and the TMA copies that were issued a bounded time
            // to land before tensor and shared memory are released.
            long long t0 = clock64();
            while (clock64() - t0 < 200000000LL) {}
        }
        __syncthreads();
    }
    if (warp == 2) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(tmem_cols));
    }
}

// ---------------------------------------------------------------------------
// CTA-pair variant for nb = 256: one cluster of two CTAs (on two SMs) owns a
// whole 256 x 256 output tile per item.  The MMA runs with cta_group::2,
// M = 256 and N = 256: each CTA stages its own 128 rows of A(m,k) and its
// own 128 rows of A(n,k) (half of the B operand), so a CTA moves 32 KB of
// operands per k-step instead of 48 KB (TF32X3) -- a third less L2 traffic
// per product, and a 6-deep ring in the same shared memory.  Tensor memory
// of each CTA holds its 128 output rows (two accumulators of 256 columns).
//   rank 0 (leader) : producer, MMA issuer, epilogue of rows 0..127;
//   rank 1          : producer, epilogue of rows 128..255.
// Both producers' TMA loads complete on the leader's full barrier (the
// .cta_group::2 form of the load); the leader's commits arrive on the empty
// and accumulator-full barriers of both CTAs (tcgen05.commit multicast);
// both epilogues release an accumulator on the leader's barrier.  The pair
// meets at cluster barriers after the barriers are initialised and before
// tensor memory is freed; every loop in between ends (waits are bounded),
// so both CTAs always reach them.
// ---------------------------------------------------------------------------
template <int MODE>
struct PairGeo {
    using G = Geo<MODE>;
    // per part: 128 rows of A(m,k) and 128 rows of A(n,k), BK columns each
    static constexpr int STAGE = G::PARTS * 2 * G::A_BYTES;   // 32 KB, BF16X6 48 KB
    static constexpr int EPI_BUFS = MODE == MODE_TF32X3 || MODE == MODE_BF16X6 ? 1 : 2;
    static constexpr int STAGES = MODE == MODE_TF32X3 ? 6 : MODE == MODE_BF16X6 ? 4 : 5;
    static constexpr int SMEM = STAGES * STAGE +
                                TC_EPI_WARPS * EPI_BUFS * TC_EPI_BUF_BYTES + 1024;
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the variable at `p` in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];"
                 :: "r"(cluster_addr) : "memory");
}

__device__ __forceinline__ bool mbar_try_cluster(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Bounded wait with cluster-scope acquire (barriers that CTAs of the pair
// arrive on): false after ~2 s or when this CTA already gave up.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity,
                                                  volatile int *abort_flag)
{
    long long t0 = clock64();
    while (!mbar_try_cluster(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > 4000000000LL) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

// TMA load into this CTA's shared memory whose completion is counted on the
// barrier at shared::cluster address `bar` (the leader's)
__device__ __forceinline__ void tma_load_4d_pair(void *dst, const CUtensorMap *map,
                                                 uint32_t bar, int c0, int c1, int c2,
                                                 int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];"
        :: "r"(smem_u32(dst)), "l"(map), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

template <int MODE>
__device__ __forceinline__ void mma_pair(uint32_t tmem, uint64_t a, uint64_t b,
                                         uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    if (!Geo<MODE>::HALF16)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, "
            "{%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}"
            :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, "
            "{%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}"
            :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z));
}

// arrive on the barrier at this offset in both CTAs of the pair once the
// MMAs issued so far are complete
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar)
{
    const uint16_t mask = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" :: "r"(smem_u32(bar)), "h"(mask) : "memory");
}

__device__ __forceinline__ uint32_t instr_desc_pair(int mode)
{
    uint32_t fmt = mode == MODE_BF16 || mode == MODE_BF16X6 ? 1u : 2u;
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (1u << 15) | (1u << 16) |
           ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
}

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TC_THREADS, 1)
k_update_pair(const __grid_constant__ CUtensorMap opmap,
              const __grid_constant__ CUtensorMap cmap, TcArgs g,
              plasma_devstat_t *st)
{
    using G = Geo<MODE>;
    using P = PairGeo<MODE>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int STAGES = P::STAGES;
    constexpr int EPI_BUFS = P::EPI_BUFS;
    constexpr int NB = 256;
    __shared__ uint64_t full_bar[STAGES], empty_bar[STAGES];
    __shared__ uint64_t tfull_bar[2], tempty_bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ int go_s;
    __shared__ volatile int abort_s;

    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    // items: whole tiles; g.ipc tiles per pair, g.nitems tiles in all
    const long long pair = blockIdx.x >> 1;
    const long long first = pair * g.ipc;
    if (first >= g.nitems) return;                 // the same for both CTAs
    const int nit = (int)min((long long)g.ipc, g.nitems - first);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *stage_base =
        (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    // stage: the PARTS parts of 128 rows of A(m,k), then those of A(n,k)
    constexpr int HALF = G::A_BYTES;
    constexpr int STAGE_BYTES = P::STAGE;
    constexpr int nkb = NB / G::BK;
    constexpr uint32_t tmem_cols = 2 * NB;

    if (tid == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull_bar[a], 1);
            mbar_init(&tempty_bar[a], 2 * TC_EPI_WARPS);
        }
        abort_s = 0;
        go_s = !plasma_failed(st);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    cluster_sync_all();                            // barriers of both CTAs ready
    // the leader's view of the device status decides for the pair
    int go;
    {
        const uint32_t a = peer_addr((const void *)&go_s, 0);
        asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(go) : "r"(a) : "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base_s)), "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;
    const uint32_t full_lead0 = peer_addr(&full_bar[0], 0);   // leader's full_bar[0]
    const uint32_t tempty_lead0 = peer_addr(&tempty_bar[0], 0);

    if (!go) {
        // status already failed: no work, both CTAs go to the teardown
    } else if (warp == 0 && lane == 0) {
        // ---------------- producer (both CTAs)
        int it = 0;
        bool ok = true;
        for (int j = 0; j < nit && ok; j++) {
            int m, n, si;
            tc_item(g, 2 * (first + j) + rank, m, n, si);
            const int row0 = (int)rank * TC_M;   // this CTA's rows of both operands
            for (int kb = 0; kb < nkb; kb++, it++) {
                const int s = it % STAGES;
                if (it >= STAGES &&
                    !mbar_wait_cluster(&empty_bar[s], ((it / STAGES) - 1) & 1, &abort_s)) {
                    ok = false;
                    break;
                }
                unsigned char *sp = stage_base + s * STAGE_BYTES;
                const uint32_t fb = full_lead0 + (uint32_t)(s * sizeof(uint64_t));
                if (leader) mbar_expect_tx(&full_bar[s], 2u * (uint32_t)STAGE_BYTES);
#pragma unroll
                for (int p = 0; p < G::PARTS; p++) {
                    const int toff = g.poff + p * g.mt;
                    tma_load_4d_pair(sp + p * HALF, &opmap, fb, 0, kb * G::BK,
                                     row0 / G::MNBOX, m + toff);
                    tma_load_4d_pair(sp + (G::PARTS + p) * HALF, &opmap, fb, 0, kb * G::BK,
                                     row0 / G::MNBOX, n + toff);
                }
            }
        }
    } else if (warp == 1 && lane == 0 && leader) {
        // ---------------- MMA issuer (leader only)
        const uint32_t idesc = instr_desc_pair(MODE);
        int it = 0;
        bool ok = true;
        for (int j = 0; j < nit && ok; j++) {
            const int a = j & 1;
            if (j >= 2 && !mbar_wait_cluster(&tempty_bar[a], ((j >> 1) - 1) & 1, &abort_s))
                break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc_t = tmem + (uint32_t)(a * NB);
            for (int kb = 0; kb < nkb; kb++, it++) {
                const int s = it % STAGES;
                if (!mbar_wait_cluster(&full_bar[s], (it / STAGES) & 1, &abort_s)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                unsigned char *sp = stage_base + s * STAGE_BYTES;
                unsigned char *sa_hi = sp;
                unsigned char *sb_hi = sp + G::PARTS * HALF;
#pragma unroll
                for (int kk = 0; kk < G::BK / G::KI; kk++) {
                    const uint32_t acc_on = (kb | kk) != 0;
                    uint64_t da = smem_desc(sa_hi + kk * G::KI * 128, G::CHUNK, G::SBO,
                                            G::LAYOUT);
                    uint64_t db = smem_desc(sb_hi + kk * G::KI * 128, G::CHUNK, G::SBO,
                                            G::LAYOUT);
                    if (MODE == MODE_TF32X3) {
                        uint64_t dal = smem_desc(sa_hi + HALF + kk * G::KI * 128, G::CHUNK,
                                                 G::SBO, G::LAYOUT);
                        uint64_t dbl = smem_desc(sb_hi + HALF + kk * G::KI * 128, G::CHUNK,
                                                 G::SBO, G::LAYOUT);
                        mma_pair<MODE>(acc_t, dal, db, idesc, acc_on);
                        mma_pair<MODE>(acc_t, da, dbl, idesc, 1u);
                        mma_pair<MODE>(acc_t, da, db, idesc, 1u);
                    } else if (MODE == MODE_BF16X6) {
                        // parts h, m, l at offsets 0, HALF, 2 HALF; small terms first
                        uint64_t dam = smem_desc(sa_hi + HALF + kk * G::KI * 128, G::CHUNK,
                                                 G::SBO, G::LAYOUT);
                        uint64_t dal = smem_desc(sa_hi + 2 * HALF + kk * G::KI * 128,
                                                 G::CHUNK, G::SBO, G::LAYOUT);
                        uint64_t dbm = smem_desc(sb_hi + HALF + kk * G::KI * 128, G::CHUNK,
                                                 G::SBO, G::LAYOUT);
                        uint64_t dbl = smem_desc(sb_hi + 2 * HALF + kk * G::KI * 128,
                                                 G::CHUNK, G::SBO, G::LAYOUT);
                        mma_pair<MODE>(acc_t, dal, db, idesc, acc_on);
                        mma_pair<MODE>(acc_t, da, dbl, idesc, 1u);
                        mma_pair<MODE>(acc_t, dam, dbm, idesc, 1u);
                        mma_pair<MODE>(acc_t, dam, db, idesc, 1u);
                        mma_pair<MODE>(acc_t, da, dbm, idesc, 1u);
                        mma_pair<MODE>(acc_t, da, db, idesc, 1u);
                    } else {
                        mma_pair<MODE>(acc_t, da, db, idesc, acc_on);
                    }
                }
                mma_commit_pair(&empty_bar[s]);
            }
            if (ok) mma_commit_pair(&tfull_bar[a]);
        }
    } else if (warp >= TC_EPI_WARP0) {
        // ---------------- epilogue (both CTAs): this CTA's 128 rows
        const int e = warp - TC_EPI_WARP0;
        const int q = warp & 3;
        const int half = e / 4;
        float *stage_epi = (float *)(stage_base + STAGES * STAGE_BYTES) +
                           (size_t)e * EPI_BUFS * (TC_EPI_BUF_BYTES / 4);
        int nchunk = 0;
        for (int j = 0; j < nit; j++) {
            const int a = j & 1;
            const bool ok = __all_sync(0xffffffffu,
                                       mbar_wait_cluster(&tfull_bar[a], (j >> 1) & 1, &abort_s));
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int m, n, si;
            tc_item(g, 2 * (first + j) + rank, m, n, si);
            const int tile = (int)(((const char *)plasma_tile_addr(g.A, m, n) -
                                    (const char *)g.A.matrix) / ((size_t)NB * NB * 4));
            const int r0 = si * TC_M + 32 * q;
            const int row = r0 + lane;
            const bool diag = m == n;
            const int c0 = half * (NB / 2);
            for (int cc = c0; cc < c0 + NB / 2; cc += 32, nchunk++) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * NB + cc), v);
                float *buf = stage_epi + (nchunk % EPI_BUFS) * (TC_EPI_BUF_BYTES / 4);
                if (nchunk >= EPI_BUFS && lane == 0) bulk_wait_read<EPI_BUFS - 1>();
                __syncwarp();
#pragma unroll
                for (int jj = 0; jj < 32; jj++) {
                    const int col = cc + jj;
                    buf[jj * 32 + lane] = (!diag || row >= col) ? -v[jj] : 0.f;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    tma_reduce_add_3d(&cmap, buf, r0, cc, tile);
                    bulk_commit();
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(tempty_lead0 + (uint32_t)(a * sizeof(uint64_t)));
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
            long long t0 = clock64();
            while (clock64() - t0 < 200000000LL) {}
        }
        __syncthreads();
    }
    // neither CTA frees tensor memory or leaves while the pair's MMAs,
    // commits or remote arrivals may still touch it
    cluster_sync_all();
    if (warp == 2) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(tmem_cols));
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Operand map: 4-D over the column-major panel tiles
//   dim 0: 128 bytes of a column (MN inner), dim 1: K (columns, stride nb),
//   dim 2: 128-byte MN chunks (stride 128 bytes), dim 3: tiles
// so one box {128 B, BK, 128 rows / chunk, 1} lands as consecutive MN chunks
// of BK x 128 bytes, the layout the MMA descriptors describe.
bool encode_tile_map(CUtensorMap *map, void *base, CUtensorMapDataType dt,
                     int esz, int nb, long long ntiles, int bk, CUtensorMapSwizzle swz)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr) return false;
    const int mnbox = 128 / esz;
    cuuint64_t dims[4] = {(cuuint64_t)mnbox, (cuuint64_t)nb, (cuuint64_t)(nb / mnbox),
                          (cuuint64_t)ntiles};
    cuuint64_t strides[3] = {(cuuint64_t)nb * esz, 128, (cuuint64_t)nb * nb * esz};
    cuuint32_t box[4] = {(cuuint32_t)mnbox, (cuuint32_t)bk, (cuuint32_t)(TC_M / mnbox), 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(map, dt, 4, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// C map: the FP32 tiles of the descriptor, {rows, columns, tile}, box 32 x 32.
bool encode_c_map(CUtensorMap *map, const plasma_desc_t &A)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr) return false;
    const size_t tile_bytes = (size_t)A.mb * A.nb * 4;
    const long long ntiles = (long long)(plasma_desc_storage_bytes(A) / tile_bytes);
    if (ntiles <= 0) return false;
    cuuint64_t dims[3] = {(cuuint64_t)A.mb, (cuuint64_t)A.nb, (cuuint64_t)ntiles};
    cuuint64_t strides[2] = {(cuuint64_t)A.mb * 4, (cuuint64_t)tile_bytes};
    cuuint32_t box[3] = {32, 32, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, A.matrix, dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int MODE>
void launch_update(cudaStream_t s, const CUtensorMap &map, const CUtensorMap &cmap,
                   const TcArgs &g, unsigned grid, plasma_devstat_t *st)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_update_tc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Geo<MODE>::SMEM);
    }
    k_update_tc<MODE><<<grid, TC_THREADS, Geo<MODE>::SMEM, s>>>(map, cmap, g, st);
}

template <int MODE>
void launch_pair(cudaStream_t s, const CUtensorMap &map, const CUtensorMap &cmap,
                 const TcArgs &g, unsigned grid, plasma_devstat_t *st)
{
    static unsigned long long attr = 0;
    if (plasma_first_on_device(&attr)) {
        cudaFuncSetAttribute(k_update_pair<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             PairGeo<MODE>::SMEM);
    }
    k_update_pair<MODE><<<grid, TC_THREADS, PairGeo<MODE>::SMEM, s>>>(map, cmap, g, st);
}

// Items per CTA (one CTA per SM) with the smallest estimated makespan,
// waves * (ipc + 1/2) items -- a CTA's pipeline fill and its last,
// unoverlapped epilogue cost about half an item -- ties to the larger ipc.
// `unit` CTAs share an item (1, or 2 for the CTA pairs).
long long choose_ipc(long long nitems, int unit, long long sms, int max_items)
{
    long long best_ipc = 1, best_cost = -1;
    for (long long ipc = 1; ipc <= max_items; ipc++) {
        const long long ctas = unit * ((nitems + ipc - 1) / ipc);
        const long long cost = ((ctas + sms - 1) / sms) * (2 * ipc + 1);
        if (best_cost < 0 || cost <= best_cost) {
            best_cost = cost;
            best_ipc = ipc;
        }
    }
    return best_ipc;
}

}  // namespace

// Layout of the rounded panel copies.  full = 0: one panel per buffer (the
// caller alternates two), row tile m of the panel at tile m, part p at
// + p * mt.  full = 1: every panel of the factor, row tile m of panel k at
// k*mt - k(k-1)/2 + (m - k) (packed lower order), part p at + p * T with
// T = mt(mt+1)/2 -- the storage a trailing update that lags behind the
// panel stream reads from.
namespace {
void panel_layout(const plasma_desc_t &A, int k, int full, int *poff, int *pstride)
{
    const int mt = A.mt;
    if (!full) {
        *poff = 0;
        *pstride = mt;
    } else {
        *poff = k * mt - k * (k - 1) / 2 - k;
        *pstride = mt * (mt + 1) / 2;
    }
}

int mode_parts(int mode)
{
    return mode == PLASMA_TC_TF32X3 ? 2 : mode == PLASMA_TC_BF16X6 ? 3 : 1;
}
}  // namespace

extern "C" void plasma_cuda_panel_layout(plasma_desc_t A, int k, int full, int *poff,
                                         int *pstride)
{
    panel_layout(A, k, full, poff, pstride);
}

// Eligibility of the tensor-core update for an FP32 descriptor: general or
// packed-lower storage, lower, square tiles of 128 or 256, no ragged tile.
extern "C" int plasma_cuda_update_tc_ok(plasma_desc_t A, plasma_enum_t uplo)
{
    return A.precision == PlasmaRealFloat &&
           (A.type == PlasmaGeneral || A.type == PlasmaLower) &&
           uplo == PlasmaLower && A.mb == A.nb && (A.mb == 128 || A.mb == 256) &&
           A.gm % A.mb == 0 && A.gn % A.nb == 0 && A.i == 0 && A.j == 0;
}

// Bytes of the operand copies (plasma_cuda_panel_round): one panel
// (full = 0) or all panels of the factor (full = 1).
extern "C" size_t plasma_cuda_panel_bytes(int mode, plasma_desc_t A, int full)
{
    if (mode < PLASMA_TC_TF32 || mode > PLASMA_TC_BF16X6) return 0;
    int poff, pstride;
    panel_layout(A, 0, full, &poff, &pstride);
    const size_t esz = mode == PLASMA_TC_BF16 || mode == PLASMA_TC_BF16X6 ? 2 : 4;
    return (size_t)mode_parts(mode) * pstride * A.mb * A.mb * esz;
}

// The operands come from `panel`: the copy of panel k made by
// plasma_cuda_panel_round for the same mode and layout (`full`), 1024-byte
// aligned.  Returns 0 (nothing launched) when the update is not eligible.
extern "C" int plasma_cuda_update_tc(cudaStream_t s, plasma_devstat_t *st,
                                     int mode, plasma_desc_t A, int k, int nlo,
                                     int nhi, const void *panel, int full, int num_sms)
{
    if (nhi <= nlo) return 1;
    const int nb = A.mb;
    long long tiles = 0;
    for (int n = nlo; n < nhi; n++) tiles += A.mt - n;
    const long long nitems = tiles * (nb / TC_M);
    if (nitems <= 0) return 1;
    if (panel == nullptr || ((uintptr_t)panel & 1023) != 0 ||
        ((uintptr_t)A.matrix & 15) != 0)
        return 0;

    int poff, pstride;
    panel_layout(A, k, full, &poff, &pstride);
    const long long ntiles = (long long)mode_parts(mode) * pstride;
    CUtensorMap map, cmap;
    bool enc;
    switch (mode) {
    case PLASMA_TC_TF32:
        enc = encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, nb,
                              ntiles, Geo<MODE_TF32>::BK, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B);
        break;
    case PLASMA_TC_TF32X3:
        enc = encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, nb,
                              ntiles, Geo<MODE_TF32X3>::BK,
                              CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B);
        break;
    case PLASMA_TC_BF16:
        enc = encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, nb,
                              ntiles, Geo<MODE_BF16>::BK, CU_TENSOR_MAP_SWIZZLE_128B);
        break;
    case PLASMA_TC_BF16X6:
        if (nb != 2 * TC_M) return 0;                 // CTA-pair kernel only
        enc = encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, nb,
                              ntiles, Geo<MODE_BF16X6>::BK, CU_TENSOR_MAP_SWIZZLE_128B);
        break;
    default:
        return 0;
    }
    if (!enc || !encode_c_map(&cmap, A))
        return 0;

    TcArgs g;
    g.A = A;
    g.k = k;
    g.nlo = nlo;
    g.nhi = nhi;
    g.poff = poff;
    g.mt = pstride;
    // PLASMA_UPDATE_MAX_ITEMS caps the items per CTA (default 8): shorter
    // CTAs hand SMs back to the panel stream sooner.  PLASMA_UPDATE_PAIR
    // selects the CTA-pair kernel for 256-wide tiles (default on; 0 = off).
    static int max_items = -1, pair_mode = -1;
    if (max_items < 0) {
        const char *env = getenv("PLASMA_UPDATE_MAX_ITEMS");
        max_items = env ? atoi(env) : 8;
        if (max_items < 1 || max_items > 64) max_items = 8;
        env = getenv("PLASMA_UPDATE_PAIR");
        pair_mode = env ? atoi(env) != 0 : 1;
    }
    const long long sms = num_sms > 0 ? num_sms : 148;
    const bool use_pair = (pair_mode || mode == PLASMA_TC_BF16X6) && nb == 2 * TC_M;
    unsigned grid;
    if (use_pair) {
        g.nitems = tiles;
        g.ipc = (int)choose_ipc(tiles, 2, sms, max_items);
        grid = (unsigned)(2 * ((tiles + g.ipc - 1) / g.ipc));
    } else {
        g.nitems = nitems;
        g.ipc = (int)choose_ipc(nitems, 1, sms, max_items);
        grid = (unsigned)((nitems + g.ipc - 1) / g.ipc);
    }

    PLASMA_COUNT_LAUNCH();
    double flops = 0.0, bytes = 0.0;
    for (int n = nlo; n < nhi; n++) {
        double cn = plasma_tile_mview(A, n), K = nb;
        for (int m = n; m < A.mt; m++) {
            double rm = plasma_tile_mview(A, m);
            flops += (m == n) ? cn * (cn + 1) * K : 2.0 * rm * cn * K;
            bytes += 4.0 * (m == n ? cn * (cn + 1) : 2.0 * rm * cn);
        }
    }
    int prof = plasma_prof_begin(s);
    if (use_pair) {
        switch (mode) {
        case PLASMA_TC_TF32: launch_pair<MODE_TF32>(s, map, cmap, g, grid, st); break;
        case PLASMA_TC_TF32X3: launch_pair<MODE_TF32X3>(s, map, cmap, g, grid, st); break;
        case PLASMA_TC_BF16X6: launch_pair<MODE_BF16X6>(s, map, cmap, g, grid, st); break;
        default: launch_pair<MODE_BF16>(s, map, cmap, g, grid, st); break;
        }
    } else {
        switch (mode) {
        case PLASMA_TC_TF32: launch_update<MODE_TF32>(s, map, cmap, g, grid, st); break;
        case PLASMA_TC_TF32X3: launch_update<MODE_TF32X3>(s, map, cmap, g, grid, st); break;
        default: launch_update<MODE_BF16>(s, map, cmap, g, grid, st); break;
        }
    }
    plasma_prof_end(prof, s, PLASMA_KCLASS_UPDATE, flops, bytes);
    return 1;
}

// Operand copy of panel k: panel tile m (m = k+1 .. mt-1) <- A(m,k) rounded
// to the product precision, same column-major layout.  TF32: round to
// nearest, ties away, kept in an FP32 container; BF16: round to nearest
// even; TF32X3: hi = tf32(a) at tile m and lo = tf32(a - hi) at tile m + mt
// (a - hi is exact in FP32).
namespace {
template <int MODE>
__global__ void k_panel_round(plasma_desc_t A, int k, void *panel, int poff, int pstride,
                              const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int m = k + 1 + blockIdx.y;
    const int nb = A.mb;
    const float4 *a = (const float4 *)plasma_tile_addr(A, m, k);
    const size_t tot = (size_t)nb * nb;
    const size_t t = (size_t)poff + m;          // operand tile of row m
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot / 4;
         e += (size_t)gridDim.x * blockDim.x) {
        const float4 x = a[e];
        const float xs[4] = {x.x, x.y, x.z, x.w};
        if (MODE == MODE_BF16) {
            __nv_bfloat16 *o = (__nv_bfloat16 *)panel + t * tot + 4 * e;
#pragma unroll
            for (int i = 0; i < 4; i++) o[i] = __float2bfloat16_rn(xs[i]);
        } else if (MODE == MODE_BF16X6) {
            // h, m, l planes at tiles m, m + mt, m + 2 mt; both differences
            // are exact in FP32 (each drops the leading 8 significant bits)
            __nv_bfloat16 *o = (__nv_bfloat16 *)panel + t * tot + 4 * e;
            const size_t plane = (size_t)pstride * tot;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const __nv_bfloat16 h = __float2bfloat16_rn(xs[i]);
                const float r1 = xs[i] - __bfloat162float(h);
                const __nv_bfloat16 md = __float2bfloat16_rn(r1);
                const float r2 = r1 - __bfloat162float(md);
                o[i] = h;
                o[plane + i] = md;
                o[2 * plane + i] = __float2bfloat16_rn(r2);
            }
        } else {
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi[i]) : "f"(xs[i]));
                if (MODE == MODE_TF32X3) {
                    float r = xs[i] - __uint_as_float(hi[i]);
                    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo[i]) : "f"(r));
                }
            }
            uint4 *o = (uint4 *)panel + (t * tot) / 4 + e;
            *o = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            if (MODE == MODE_TF32X3) {
                uint4 *ol = (uint4 *)panel + ((t + pstride) * tot) / 4 + e;
                *ol = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            }
        }
    }
}
}  // namespace

extern "C" void plasma_cuda_panel_round(cudaStream_t s, plasma_devstat_t *st,
                                        int mode, plasma_desc_t A, int k,
                                        void *panel, int full)
{
    int rows = A.mt - k - 1;
    if (rows <= 0) return;
    int poff, pstride;
    panel_layout(A, k, full, &poff, &pstride);
    PLASMA_COUNT_LAUNCH();
    dim3 grid(16, rows);
    switch (mode) {
    case PLASMA_TC_BF16:
        k_panel_round<MODE_BF16><<<grid, 256, 0, s>>>(A, k, panel, poff, pstride, st);
        break;
    case PLASMA_TC_TF32X3:
        k_panel_round<MODE_TF32X3><<<grid, 256, 0, s>>>(A, k, panel, poff, pstride, st);
        break;
    case PLASMA_TC_BF16X6:
        k_panel_round<MODE_BF16X6><<<grid, 256, 0, s>>>(A, k, panel, poff, pstride, st);
        break;
    default:
        k_panel_round<MODE_TF32><<<grid, 256, 0, s>>>(A, k, panel, poff, pstride, st);
        break;
    }
}
