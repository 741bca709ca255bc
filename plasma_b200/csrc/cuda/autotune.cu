// autotune.cu -- measured tile-shape selection (the tuning tables of
// control/tuning.c).  The reference reads nb from a Lua script
// (control/tuning.c:367-374, tuning/default.lua); this library measures it
// on the GPU it runs on.
//
// plasma_autotune_potrf: for a matrix order n, times the tile factorization
//   (plasma_omp_?potrf, packed lower storage, the context's factor mode) of
//   a synthetic diagonally dominant SPD matrix for every candidate tile size
//   nb in {128, 256, 384, 512} (those not above max(n, 128)), two runs each,
//   CUDA events on the context stream; the fastest nb goes into the table
//   for n's size bucket.
// plasma_autotune_batched: for every size bucket of the batched kernels
//   (orders 32, 64, 128, 256, 512), times a batch of `count` matrices of the
//   bucket's largest order with block widths 16 and 32; the faster goes
//   into the batched table.
#include "common.cuh"

namespace {

// a_ij = u(max(i,j), min(i,j)) in [-0.5, 0.5) off the diagonal, n + u on it
__device__ __forceinline__ double spd_entry(int i, int j, int n, unsigned seed)
{
    const int r = max(i, j), c = min(i, j);
    unsigned long long h = ((unsigned long long)r * 0x9E3779B97F4A7C15ull) ^
                           ((unsigned long long)c * 0xC2B2AE3D27D4EB4Full) ^ seed;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    return i == j ? n + u : u;
}

template <typename T>
__global__ void k_fill_spd_desc(plasma_desc_t A, unsigned seed)
{
    const int i = blockIdx.y * 32 + threadIdx.x;
    const int j = blockIdx.x * 8 + threadIdx.y;
    if (i >= A.m || j >= A.n || i < j) return;       // the lower triangle is stored
    const int tm = i / A.mb, tn = j / A.nb;
    T *t = (T *)plasma_tile_addr(A, tm, tn);
    t[(size_t)(j - tn * A.nb) * plasma_tile_mmain(A, tm) + (i - tm * A.mb)] =
        (T)spd_entry(i, j, A.m, seed);
}

template <typename T>
__global__ void k_fill_spd_batch(T *A, int n, long long stride, long long count, unsigned seed)
{
    const long long tot = stride * count;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e % stride;
        if (r >= (long long)n * n) continue;
        const int i = (int)(r % n), j = (int)(r / n);
        A[e] = (T)spd_entry(i, j, n, seed + (unsigned)(e / stride));
    }
}

void fill_desc(cudaStream_t s, plasma_desc_t A, unsigned seed)
{
    dim3 grid((A.n + 7) / 8, (A.m + 31) / 32), block(32, 8);
    if (A.precision == PlasmaRealDouble)
        k_fill_spd_desc<double><<<grid, block, 0, s>>>(A, seed);
    else
        k_fill_spd_desc<float><<<grid, block, 0, s>>>(A, seed);
}

}  // namespace

extern "C" int plasma_autotune_potrf(plasma_enum_t dtyp, int n, double *best_ms)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) return PlasmaErrorNotInitialized;
    if (dtyp != PlasmaRealDouble && dtyp != PlasmaRealFloat) return -1;
    if (n <= 0) return -2;
    if (plasma->device < 0) return PlasmaErrorEnvironment;
    static const int cand[4] = {128, 256, 384, 512};
    const int cap = n > 128 ? n : 128;
    cudaStream_t s = plasma->stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 0;
    float best_t = 0.f;
    for (int c = 0; c < 4; c++) {
        const int nb = cand[c];
        if (nb > cap) break;
        plasma_desc_t A;
        if (plasma_desc_triangular_create(dtyp, PlasmaLower, nb, nb, n, n, 0, 0, n, n, &A) !=
            PlasmaSuccess)
            continue;
        float t = -1.f;
        for (int rep = 0; rep < 2; rep++) {
            fill_desc(s, A, 7u);
            plasma_sequence_t seq;
            plasma_request_t req;
            plasma_sequence_init(&seq);
            plasma_request_init(&req);
            cudaEventRecord(e0, s);
            if (dtyp == PlasmaRealDouble)
                plasma_omp_dpotrf(PlasmaLower, A, &seq, &req);
            else
                plasma_omp_spotrf(PlasmaLower, A, &seq, &req);
            cudaEventRecord(e1, s);
            if (plasma_sequence_wait(&seq) != PlasmaSuccess) {
                t = -1.f;
                break;
            }
            cudaEventElapsedTime(&t, e0, e1);
        }
        plasma_desc_destroy(&A);
        if (t >= 0.f && (best == 0 || t < best_t)) {
            best = nb;
            best_t = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best == 0) return PlasmaErrorInternal;
    plasma_tuning_set_potrf_nb(dtyp, n, best);
    if (best_ms) *best_ms = best_t;
    return best;
}

extern "C" int plasma_autotune_batched(plasma_enum_t dtyp, int count)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) return PlasmaErrorNotInitialized;
    if (dtyp != PlasmaRealDouble && dtyp != PlasmaRealFloat) return -1;
    if (count <= 0) return -2;
    if (plasma->device < 0) return PlasmaErrorEnvironment;
    const size_t elem = plasma_element_size(dtyp);
    cudaStream_t s = plasma->stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = PlasmaSuccess;
    for (int order = 32; order <= 512 && rc == PlasmaSuccess; order *= 2) {
        const long long stride = ((long long)order * order + 31) / 32 * 32;
        int *sizes = (int *)malloc(sizeof(int) * count);
        void *A = NULL, *B = NULL;
        int *info = NULL;
        if (sizes == NULL ||
            cudaMalloc(&A, (size_t)stride * count * elem) != cudaSuccess ||
            cudaMalloc(&B, (size_t)(((order + 31) / 32) * 32) * count * elem) != cudaSuccess ||
            cudaMalloc(&info, sizeof(int) * count) != cudaSuccess) {
            cudaGetLastError();
            rc = PlasmaErrorOutOfMemory;
        }
        for (int i = 0; sizes && i < count; i++) sizes[i] = order;
        float best_t = 0.f;
        int best = 0;
        for (int nb = 16; nb <= 32 && rc == PlasmaSuccess; nb *= 2) {
            plasma_tuning_set_batched_nb(dtyp, order, nb);
            plasma_batch_t *plan = NULL;
            if (plasma_batch_create(dtyp, count, sizes, &plan) != PlasmaSuccess) {
                rc = PlasmaErrorOutOfMemory;
                break;
            }
            float t = -1.f;
            for (int rep = 0; rep < 2; rep++) {
                if (dtyp == PlasmaRealDouble)
                    k_fill_spd_batch<double><<<1184, 256, 0, s>>>((double *)A, order, stride,
                                                                   count, 11u);
                else
                    k_fill_spd_batch<float><<<1184, 256, 0, s>>>((float *)A, order, stride,
                                                                  count, 11u);
                cudaMemsetAsync(B, 0, (size_t)(((order + 31) / 32) * 32) * count * elem, s);
                cudaEventRecord(e0, s);
                if (dtyp == PlasmaRealDouble)
                    plasma_dposv_batched(plan, (double *)A, (double *)B, info);
                else
                    plasma_sposv_batched(plan, (float *)A, (float *)B, info);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&t, e0, e1);
            }
            plasma_batch_destroy(plan);
            if (t >= 0.f && (best == 0 || t < best_t)) {
                best = nb;
                best_t = t;
            }
        }
        if (best) plasma_tuning_set_batched_nb(dtyp, order, best);
        free(sizes);
        cudaFree(A);
        cudaFree(B);
        cudaFree(info);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
