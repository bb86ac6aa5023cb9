// Allocation-free variant of grim_backward_error.
//
// Who needs it: callers that cannot allocate device memory at the time they ask for a
// backward error -- for example a host program whose GPU memory is entirely reserved by
// another framework's caching allocator, a latency-bound serving loop that must not
// enter the CUDA allocator between requests, or an FFI caller that has no device
// allocator of its own.  grim_backward_error takes its residual and norm scratch from
// the handle's workspace (a stream-ordered allocation the first time a size is seen);
// this entry point instead uses one fixed array in device global memory, compiled into
// the library, so it never allocates.
//
// Scratch: g_noalloc_scratch below, GRIM_NOALLOC_SCRATCH_BYTES on every device that
// loads the library, held until the process exits.  Sizes are limited to
// n <= GRIM_NOALLOC_MAX_N and nrhs <= GRIM_NOALLOC_MAX_NRHS; larger requests are
// rejected with GRIM_ERR_ARGUMENT and a message, before any GPU work.
//
// Set-up: host code cannot pass the array's name to a kernel (in host code the name is
// only a host-side stand-in, not a device address), so every call, with the handle's
// device current, looks the device address up with cudaGetSymbolAddress (cheap) and
// checks the result.  Looking it up per call, not caching it, keeps the address valid
// if the device's context is torn down and recreated between calls.  The first lookup on
// a device may load the library's module there, so make the first call on each device
// before any stream capture on it.
//
// Sharing: every call on a device uses the same array and leaves its contents behind.
// Each call writes every scratch word before reading it (the residual starts as a copy
// of B, every partial sum is stored before it is summed), so nothing needs clearing;
// but two calls whose GPU work overlaps (different streams, threads or handles on the
// same device) race on the array and must be serialized by the caller.
#include <cuda_runtime.h>

#define GRIM_NOALLOC_MAX_N 1024
#define GRIM_NOALLOC_MAX_NRHS 128

// Layout (bytes): residual R (n x nrhs complex128) | row partials (ROWSUM_CHUNKS x n
// doubles) | row sums (n doubles) | column maxima (3 x nrhs doubles) | scalars (8 doubles)
#define NOALLOC_R_BYTES ((size_t)GRIM_NOALLOC_MAX_N * GRIM_NOALLOC_MAX_NRHS * 16)
#define NOALLOC_PART_BYTES ((size_t)ROWSUM_CHUNKS * GRIM_NOALLOC_MAX_N * 8)
#define NOALLOC_ROW_BYTES ((size_t)GRIM_NOALLOC_MAX_N * 8)
#define NOALLOC_COL_BYTES ((size_t)3 * GRIM_NOALLOC_MAX_NRHS * 8)
#define NOALLOC_SCALAR_BYTES ((size_t)8 * 8)
#define GRIM_NOALLOC_SCRATCH_BYTES \
    (NOALLOC_R_BYTES + NOALLOC_PART_BYTES + NOALLOC_ROW_BYTES + NOALLOC_COL_BYTES + NOALLOC_SCALAR_BYTES)

static __device__ __align__(256) unsigned char g_noalloc_scratch[GRIM_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on h's device, looked up on every call.
static int noalloc_scratch(grim_context *h, unsigned char **out) {
    DeviceGuard g(h->device);
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return grim_cuda_check(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    *out = (unsigned char *)p;
    return GRIM_OK;
}

template <typename TA>
static int noalloc_berr(grim_context *h, int n, int nrhs, const TA *A, int64_t lda, const double2 *X, int64_t ldx,
                        const double2 *B, int64_t ldb, double *berr, unsigned char *scratch) {
    double2 *R = (double2 *)scratch;
    double *partial = (double *)(scratch + NOALLOC_R_BYTES);
    double *rowsum = (double *)(scratch + NOALLOC_R_BYTES + NOALLOC_PART_BYTES);
    double *colmax = (double *)(scratch + NOALLOC_R_BYTES + NOALLOC_PART_BYTES + NOALLOC_ROW_BYTES);
    double *sc = (double *)(scratch + NOALLOC_R_BYTES + NOALLOC_PART_BYTES + NOALLOC_ROW_BYTES + NOALLOC_COL_BYTES);
    const int64_t ldr = n;
    // ||A||_inf into sc[0]
    dim3 g(ceil_div(n, 128), ROWSUM_CHUNKS);
    k_row_abs_partial<TA><<<g, 128, 0, h->stream>>>(n, A, lda, partial);
    GRIM_CHECK_LAUNCH(h, "k_row_abs_partial");
    k_row_abs_finish<<<ceil_div(n, 128), 128, 0, h->stream>>>(n, partial, rowsum);
    GRIM_CHECK_LAUNCH(h, "k_row_abs_finish");
    k_max_reduce<<<1, 1024, 0, h->stream>>>(n, rowsum, sc);
    GRIM_CHECK_LAUNCH(h, "k_max_reduce");
    // R = B - A X, then column maxima and the backward error
    GRIM_CHECK_CUDA(cudaMemcpy2DAsync(R, ldr * sizeof(double2), B, ldb * sizeof(double2), n * sizeof(double2), nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream));
    GRIM_TRY((gemm<double2, TA, double2, double2, true, true>(h, n, nrhs, n, A, lda, X, ldx, R, ldr)));
    k_col_absmax3<double2><<<nrhs, 256, 0, h->stream>>>(n, R, ldr, X, ldx, B, ldb, colmax);
    GRIM_CHECK_LAUNCH(h, "k_col_absmax3");
    k_berr_finish<<<1, 1024, 0, h->stream>>>(nrhs, colmax, sc, berr, nullptr, sc + 1);
    GRIM_CHECK_LAUNCH(h, "k_berr_finish");
    return GRIM_OK;
}

extern "C" int grim_backward_error_noalloc(grim_handle_t h, int n, int nrhs, const void *A, int64_t lda,
                                           int a_complex64, const void *X, int64_t ldx, const void *B, int64_t ldb,
                                           double *berr_dev) {
    if (!h || n <= 0 || nrhs <= 0 || !A || !X || !B || !berr_dev || lda < n || ldx < n || ldb < n)
        return grim_fail(GRIM_ERR_ARGUMENT, "grim_backward_error_noalloc: bad arguments");
    if (n > GRIM_NOALLOC_MAX_N || nrhs > GRIM_NOALLOC_MAX_NRHS)
        return grim_fail(GRIM_ERR_ARGUMENT,
                         "grim_backward_error_noalloc: n must be <= 1024 and nrhs <= 128 (the size of the library's "
                         "fixed scratch array); use grim_backward_error for larger systems");
    unsigned char *scratch = nullptr;
    GRIM_TRY(noalloc_scratch(h, &scratch));
    DeviceGuard g(h->device);
    if (a_complex64)
        return noalloc_berr(h, n, nrhs, (const float2 *)A, lda, (const double2 *)X, ldx, (const double2 *)B, ldb,
                            berr_dev, scratch);
    return noalloc_berr(h, n, nrhs, (const double2 *)A, lda, (const double2 *)X, ldx, (const double2 *)B, ldb,
                        berr_dev, scratch);
}
