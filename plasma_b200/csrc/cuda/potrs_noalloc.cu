// potrs_noalloc.cu -- plasma_omp_dpotrs_noalloc: the single right-hand-side
// FP64 tile potrs (forward and backward one-launch block sweeps, trsv.cu)
// with its scratch in a file-scope device array instead of memory the library
// allocates.  No reference counterpart; the computation is that of
// plasma_omp_dpotrs for one right-hand side.
//
// It serves callers that must not allocate device memory during a solve:
// a process whose device memory is already handed out to another allocator
// (a framework's caching pool that holds nearly all of HBM, a service with a
// fixed, pre-planned footprint), and a latency-bound solve loop, where
// cudaMalloc/cudaFree would synchronise the device and stall the work of
// other streams.  The library's plain potrs grows its workspace with
// cudaMalloc on first use at a new size; this entry point never does.
//
// Scratch: the inverses of the 64 x 64 diagonal blocks of the factor
// (64 * 64 doubles per block, PLASMA_NOALLOC_MAX_N / 64 blocks = 4 MiB) and
// the sweep's ticket, abort word and per-block ready flags (4 KiB).  The
// first call on a device looks the array's address up with
// cudaGetSymbolAddress; that first call belongs before any stream capture.
// Every call overwrites the array, so calls that overlap (other streams,
// other host threads) race, and the array keeps the last call's contents.
// The ticket and abort words are cleared on the stream at the start of each
// sweep; the ready flags are never cleared, each sweep waits for its own
// epoch (a per-device counter, never 0, and the array starts zeroed), and the
// block inverses are rewritten in full by every call.  The epoch counter is
// host state shared by every call on the device too: calls from several host
// threads race on it as they race on the array.
#include "common.cuh"

namespace {

constexpr int NA_SB = 64;                                  // FP64 sweep block
constexpr int NA_MAX_BLK = PLASMA_NOALLOC_MAX_N / NA_SB;
constexpr size_t NA_W_DOUBLES = (size_t)NA_MAX_BLK * NA_SB * NA_SB;
constexpr size_t NA_SYNC_BYTES = 4096;
constexpr int NA_MAX_DEVICES = 64;

__device__ __align__(256) double
    g_potrs_scratch[NA_W_DOUBLES + NA_SYNC_BYTES / sizeof(double)];

double *g_scratch_addr[NA_MAX_DEVICES];
unsigned g_epoch[NA_MAX_DEVICES];

// The sweeps compare ready flags with the epoch for equality only, so the
// counter's bit pattern is passed as it is; it skips 0 (the value of flags
// no sweep has written) when it wraps after 2^32 sweeps.
int next_epoch(int dev)
{
    if (++g_epoch[dev] == 0u)
        g_epoch[dev] = 1u;
    return (int)g_epoch[dev];
}

}  // namespace

extern "C" void plasma_omp_dpotrs_noalloc(plasma_enum_t uplo, plasma_desc_t A,
                                          plasma_desc_t B,
                                          plasma_sequence_t *sequence,
                                          plasma_request_t *request)
{
    plasma_context_t *plasma = plasma_context_self();
    if (plasma == NULL) {
        plasma_error("PLASMA not initialized");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (sequence == NULL || request == NULL) {
        plasma_error("NULL sequence or request");
        return;
    }
    if (uplo != PlasmaUpper && uplo != PlasmaLower) {
        plasma_error("illegal value of uplo");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (plasma_desc_check(A) != PlasmaSuccess) {
        plasma_error("invalid A");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (plasma_desc_check(B) != PlasmaSuccess) {
        plasma_error("invalid B");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (sequence->status != PlasmaSuccess)
        return;
    if (A.n == 0 || B.n == 0)
        return;
    if (plasma->device < 0 || plasma->device >= NA_MAX_DEVICES) {
        plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
        return;
    }
    if (A.precision != PlasmaRealDouble || B.precision != PlasmaRealDouble) {
        plasma_error("plasma_omp_dpotrs_noalloc: A and B must be double");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return;
    }
    if (A.m != A.n || B.m != A.m) {
        plasma_error("plasma_omp_dpotrs_noalloc: A must be n x n and B n x 1");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    if (A.m > PLASMA_NOALLOC_MAX_N) {
        plasma_error("plasma_omp_dpotrs_noalloc: n exceeds the static scratch "
                     "limit PLASMA_NOALLOC_MAX_N = 8192");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }
    /* one contiguous right-hand side, 64-row sweep blocks */
    if (B.n != 1 || B.nt != 1 || B.i != 0 || B.j != 0 || B.gn != 1 ||
        B.mb != A.mb || plasma_cuda_trsv_block(A) != NA_SB) {
        plasma_error("plasma_omp_dpotrs_noalloc: needs one right-hand side "
                     "(B n x 1) and square tiles with nb a multiple of 64");
        plasma_request_fail(sequence, request, PlasmaErrorNotSupported);
        return;
    }
    const int nblk = (A.m + NA_SB - 1) / NA_SB;
    if (plasma_cuda_trsv_sync_bytes(nblk) > NA_SYNC_BYTES) {
        plasma_error("plasma_omp_dpotrs_noalloc: sweep flags exceed the "
                     "static scratch");
        plasma_request_fail(sequence, request, PlasmaErrorIllegalValue);
        return;
    }

    const int dev = plasma->device;
    if (g_scratch_addr[dev] == NULL) {
        // the array's host-side name is not a device address: look the
        // address up once per device, with that device current
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);
        double *p = NULL;
        cudaError_t rc = cudaGetSymbolAddress((void **)&p, g_potrs_scratch);
        if (cur != dev && cur >= 0) cudaSetDevice(cur);
        if (rc != cudaSuccess || p == NULL) {
            cudaGetLastError();
            plasma_error("plasma_omp_dpotrs_noalloc: cudaGetSymbolAddress of "
                         "the static scratch failed");
            plasma_request_fail(sequence, request, PlasmaErrorEnvironment);
            return;
        }
        g_scratch_addr[dev] = p;
    }
    double *W = g_scratch_addr[dev];
    void *sync = W + NA_W_DOUBLES;

    plasma_call_begin(plasma, sequence, request);
    // (the checks above make A eligible for 64-row FP64 block sweeps, so
    // both sweeps launch; a sweep that does not launch fails the request)
    plasma_cuda_trtri_blocks(plasma->stream, plasma->dstat, uplo, A, W);
    if (!plasma_cuda_trsv(plasma->stream, plasma->dstat, uplo, 0, A, W, B.matrix,
                          sync, next_epoch(dev), plasma->num_sms) ||
        !plasma_cuda_trsv(plasma->stream, plasma->dstat, uplo, 1, A, W, B.matrix,
                          sync, next_epoch(dev), plasma->num_sms)) {
        plasma_error("plasma_omp_dpotrs_noalloc: the block sweep did not launch");
        plasma_request_fail(sequence, request, PlasmaErrorInternal);
    }
}
