// update_tc.cu -- trailing update of the low-precision Cholesky on the
// fifth-generation tensor cores (tcgen05, accumulators in tensor memory).
//
//     C(m,n) -= A(m,k) * A(n,k)^T     C in FP32, operands TF32 or BF16
//
// This is the SYRK/GEMM part of plasma_pspotrf (the FP32 tile Cholesky that
// the reference runs inside dsposv, compute/zcposv.c:452 ->
// compute/pzpotrf.c:57-77) with the products formed at reduced precision and
// accumulated in FP32.
//
// One CTA computes a 128 x nb block (nb = 256 or 128) of one output tile:
//   warp 0     : TMA producer -- 3-D tensor maps over the column-major tiles
//                of the rounded panel copy (128-byte swizzle; 32-byte swizzle
//                atoms for TF32, the only MN-major TF32 layout), two-stage
//                ring of 48 KB stages, plus an L2 prefetch of the C block;
//   warp 1     : MMA issuer -- one thread issues tcgen05.mma (M = 128,
//                N = nb, MN-major A and B straight from the column-major
//                tiles), tcgen05.commit frees a stage / signals the end;
//   warps 2-9  : epilogue -- tcgen05.ld of the accumulator, C -= P on FP32
//                tiles in global memory (coalesced along rows), masking the
//                strict upper triangle of diagonal tiles.
// Two CTAs share an SM, so one CTA's HBM-bound epilogue overlaps the other's
// MMAs.  Every mbarrier wait is bounded (about a second); on expiry the CTA
// records PlasmaErrorInternal, drains what it issued and frees its TMEM.
#include "common.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

namespace {

constexpr int TC_M = 128;
constexpr int TC_THREADS = 320;          // 10 warps
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_STAGE_BYTES = 48 * 1024;
constexpr int TC_STAGES = 2;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024 + 256;

enum { MODE_TF32 = 1, MODE_BF16 = 2 };

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// Bounded wait: false after ~1 s (or at once when the CTA already gave up).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          volatile int *abort_flag)
{
    long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > 4000000000LL) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map,
                                            uint64_t *bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cta.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];"
        :: "r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Shared-memory matrix descriptor of an MN-major operand.  BF16 uses the
// 128-byte swizzle (8 K-rows of 128 bytes per atom, layout type 2); MN-major
// TF32 operands only exist with the 128-byte swizzle of 32-byte atomicity
// (4 K-rows per atom, layout type 1).  lbo = stride between 128-byte MN
// chunks, sbo = stride between K atoms.
__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_u32(p) >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)layout << 61;
    return d;
}

__device__ __forceinline__ uint32_t instr_desc(int mode, int n)
{
    uint32_t fmt = mode == MODE_TF32 ? 2u : 1u;   // TF32 : BF16
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
    if (MODE == MODE_TF32)
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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
          "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
          "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct TcArgs {
    plasma_desc_t A;    // FP32 general descriptor holding C (and TF32 operands)
    int k, nlo, nhi;
    int op_base;        // tile index of panel tile 0 in the operand map
    int op_stride;      // tile-index step per tile row in the operand map
};

// work item -> (m, n, si); false when the item lies strictly above the
// diagonal of a diagonal tile
__device__ __forceinline__ bool tc_item(const TcArgs &g, int w, int &m, int &n, int &si)
{
    const int sb = g.A.mb / TC_M;
    int p = w / sb;
    si = w - p * sb;
    n = g.nlo;
    while (n < g.nhi && p >= g.A.mt - n) { p -= g.A.mt - n; n++; }
    if (n >= g.nhi) return false;
    m = n + p;
    return true;
}

template <int MODE>
__global__ void __launch_bounds__(TC_THREADS, 2)
k_update_tc(const __grid_constant__ CUtensorMap opmap, TcArgs g,
            plasma_devstat_t *st)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES], acc_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    if (plasma_failed(st)) return;
    int m, n, si;
    if (!tc_item(g, blockIdx.x, m, n, si)) return;

    const int nb = g.A.mb;                         // N of the MMA
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *stage_base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    // element geometry
    constexpr int ESZ = MODE == MODE_TF32 ? 4 : 2;
    constexpr int MNBOX = 128 / ESZ;              // elements per 128-byte row
    constexpr int BK = MODE == MODE_TF32 ? 32 : 64;
    constexpr int KI = MODE == MODE_TF32 ? 8 : 16; // K per instruction
    const int chunk_bytes = BK * 128;             // one MN chunk of a stage
    const int a_bytes = (TC_M / MNBOX) * chunk_bytes;
    const int stage_bytes = a_bytes + (nb / MNBOX) * chunk_bytes;
    const int nkb = g.A.nb / BK;                  // K = nb

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&acc_bar, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base_s)), "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    float *C = (float *)plasma_tile_addr(g.A, m, n);
    const int ldc = plasma_tile_mmain(g.A, m);
    const int i0 = si * TC_M;

    if (warp == 0 && lane == 0) {
        // ---------------- producer
        // warm L2 with the C block: nb columns of 128 rows (512 bytes each)
        for (int j = 0; j < nb; j++)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(C + (size_t)j * ldc + i0), "r"(TC_M * 4) : "memory");
        const int ta = g.op_base + m * g.op_stride;   // operand tile of A(m,k)
        const int tb = g.op_base + n * g.op_stride;   // operand tile of A(n,k)
        for (int kb = 0; kb < nkb; kb++) {
            int s = kb % TC_STAGES;
            if (kb >= TC_STAGES &&
                !mbar_wait(&empty_bar[s], ((kb / TC_STAGES) - 1) & 1, &abort_s))
                break;
            unsigned char *sa = stage_base + s * TC_STAGE_BYTES;
            unsigned char *sbp = sa + a_bytes;
            mbar_expect_tx(&full_bar[s], (uint32_t)stage_bytes);
            for (int c = 0; c < TC_M / MNBOX; c++)
                tma_load_3d(sa + c * chunk_bytes, &opmap, &full_bar[s],
                            i0 + c * MNBOX, kb * BK, ta);
            for (int c = 0; c < nb / MNBOX; c++)
                tma_load_3d(sbp + c * chunk_bytes, &opmap, &full_bar[s],
                            c * MNBOX, kb * BK, tb);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = instr_desc(MODE, nb);
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; kb++) {
            int s = kb % TC_STAGES;
            if (!mbar_wait(&full_bar[s], (kb / TC_STAGES) & 1, &abort_s)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            unsigned char *sa = stage_base + s * TC_STAGE_BYTES;
            unsigned char *sbp = sa + a_bytes;
#pragma unroll
            for (int kk = 0; kk < BK / KI; kk++) {
                constexpr uint32_t LAYOUT = MODE == MODE_TF32 ? 1u : 2u;
                constexpr uint32_t SBO = MODE == MODE_TF32 ? 512u : 1024u;
                uint64_t da = smem_desc(sa + kk * KI * 128, chunk_bytes, SBO, LAYOUT);
                uint64_t db = smem_desc(sbp + kk * KI * 128, chunk_bytes, SBO, LAYOUT);
                mma<MODE>(tmem, da, db, idesc, (kb | kk) != 0);
            }
            mma_commit(&empty_bar[s]);
        }
        mma_commit(&acc_bar);
    } else if (warp >= 2) {
        // ---------------- epilogue: warp -> TMEM lane quarter and column half
        const int e = warp - 2;
        const int q = warp & 3;                  // lanes 32q .. 32q+31
        const int half = e / 4;                  // columns [half*nb/2, ...)
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_bar, 0, &abort_s));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            const int row = i0 + 32 * q + lane;
            const int rows = plasma_tile_mview(g.A, m);
            const int cols = plasma_tile_mview(g.A, n);
            const bool diag = m == n;
            const int c0 = half * (nb / 2);
            for (int cc = c0; cc < c0 + nb / 2; cc += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)cc, v);
                if (row < rows) {
                    float cv[32];
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        int col = cc + j;
                        cv[j] = (col < cols && (!diag || row >= col))
                                    ? C[(size_t)col * ldc + row] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        int col = cc + j;
                        if (col < cols && (!diag || row >= col))
                            C[(size_t)col * ldc + row] = cv[j] - v[j];
                    }
                }
            }
        }
    }
    // ---------------- teardown
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_s) {
        if (tid == 0) {
            plasma_fail(st, PlasmaErrorInternal, 0);
            // Give the MMAs (the accumulator barrier) and the TMA copies that
            // were issued a bounded time to land before TMEM and shared
            // memory are released.
            long long t0 = clock64();
            while (!mbar_try(&acc_bar, 0) && clock64() - t0 < 400000000LL) {}
            t0 = clock64();
            while (clock64() - t0 < 100000000LL) {}
        }
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(256));
    }
}

// ---------------------------------------------------------------------------
// host side: tensor maps over column-major tile arrays
// ---------------------------------------------------------------------------
bool encode_tile_map(CUtensorMap *map, void *base, CUtensorMapDataType dt,
                     int esz, int nb, long long ntiles, int box_mn, int box_k,
                     CUtensorMapSwizzle swz)
{
    cuuint64_t dims[3] = {(cuuint64_t)nb, (cuuint64_t)nb, (cuuint64_t)ntiles};
    cuuint64_t strides[2] = {(cuuint64_t)nb * esz, (cuuint64_t)nb * nb * esz};
    cuuint32_t box[3] = {(cuuint32_t)box_mn, (cuuint32_t)box_k, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    // resolved through the runtime so that the library does not link the
    // driver library directly (it must load on machines without a GPU)
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (encode == nullptr) {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&encode,
                                    cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            encode = nullptr;
            return false;
        }
    }
    CUresult r = encode(map, dt, 3, base, dims, strides, box, estr,
                                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                                        swz,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

// Eligibility of the tensor-core update for an FP32 descriptor: general
// storage, lower, square tiles of 128 or 256 with no ragged tile.
extern "C" int plasma_cuda_update_tc_ok(plasma_desc_t A, plasma_enum_t uplo)
{
    return A.precision == PlasmaRealFloat &&
           (A.type == PlasmaGeneral || A.type == PlasmaLower) &&
           uplo == PlasmaLower && A.mb == A.nb && (A.mb == 128 || A.mb == 256) &&
           A.gm % A.mb == 0 && A.gn % A.nb == 0 && A.i == 0 && A.j == 0;
}

// The operands come from `panel`: the copy of panel k rounded to the product
// precision (TF32 values in FP32 containers, or BF16), tile m at
// panel + m*nb*nb elements, column-major, 1024-byte aligned.
extern "C" int plasma_cuda_update_tc(cudaStream_t s, plasma_devstat_t *st,
                                     int mode, plasma_desc_t A, int k, int nlo,
                                     int nhi, const void *panel)
{
    if (nhi <= nlo) return 1;
    const int nb = A.mb;
    long long pairs = 0;
    for (int n = nlo; n < nhi; n++) pairs += A.mt - n;
    long long nitems = pairs * (nb / TC_M);
    if (nitems <= 0) return 1;

    CUtensorMap map;
    TcArgs g;
    g.A = A;
    g.k = k;
    g.nlo = nlo;
    g.nhi = nhi;
    if (panel == nullptr || ((uintptr_t)panel & 1023) != 0)
        return 0;
    if (mode == PlasmaFactorTF32) {
        if (!encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                             nb, A.mt, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B))
            return 0;
    } else {
        if (!encode_tile_map(&map, (void *)panel, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                             nb, A.mt, 64, 64, CU_TENSOR_MAP_SWIZZLE_128B))
            return 0;
    }
    g.op_base = 0;
    g.op_stride = 1;
    static bool attr[3] = {false, false, false};
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
    if (mode == PlasmaFactorTF32) {
        if (!attr[1]) {
            cudaFuncSetAttribute(k_update_tc<MODE_TF32>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            attr[1] = true;
        }
        k_update_tc<MODE_TF32><<<(unsigned)nitems, TC_THREADS, TC_SMEM, s>>>(map, g, st);
    } else {
        if (!attr[2]) {
            cudaFuncSetAttribute(k_update_tc<MODE_BF16>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            attr[2] = true;
        }
        k_update_tc<MODE_BF16><<<(unsigned)nitems, TC_THREADS, TC_SMEM, s>>>(map, g, st);
    }
    plasma_prof_end(prof, s, PLASMA_KCLASS_UPDATE, flops, bytes);
    return 1;
}

// Operand copy of panel k: panel tile m (m = k+1 .. mt-1) <- A(m,k) rounded
// to the product precision (TF32: round to nearest, ties away, kept in an
// FP32 container; BF16: round to nearest even), same column-major layout.
namespace {
template <bool BF16>
__global__ void k_panel_round(plasma_desc_t A, int k, void *panel,
                              const plasma_devstat_t *st)
{
    if (plasma_failed(st)) return;
    const int m = k + 1 + blockIdx.y;
    const int nb = A.mb;
    const float *a = (const float *)plasma_tile_addr(A, m, k);
    const size_t tot = (size_t)nb * nb;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (size_t)gridDim.x * blockDim.x) {
        if (BF16) {
            ((__nv_bfloat16 *)panel)[(size_t)m * tot + e] = __float2bfloat16_rn(a[e]);
        } else {
            uint32_t r;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a[e]));
            ((uint32_t *)panel)[(size_t)m * tot + e] = r;
        }
    }
}
}  // namespace

extern "C" void plasma_cuda_panel_round(cudaStream_t s, plasma_devstat_t *st,
                                        int mode, plasma_desc_t A, int k,
                                        void *panel)
{
    int rows = A.mt - k - 1;
    if (rows <= 0) return;
    PLASMA_COUNT_LAUNCH();
    if (mode == PlasmaFactorBF16)
        k_panel_round<true><<<dim3(16, rows), 256, 0, s>>>(A, k, panel, st);
    else
        k_panel_round<false><<<dim3(16, rows), 256, 0, s>>>(A, k, panel, st);
}
