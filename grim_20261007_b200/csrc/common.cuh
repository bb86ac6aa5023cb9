// Shared device/host helpers for libgrimgpu: complex arithmetic on interleaved
// pairs, the handle (context) structure, error reporting, workspace.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/grimgpu.h"

// ---------------------------------------------------------------- complex math
template <typename T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };

template <typename C> struct real_of;
template <> struct real_of<double2> { using type = double; };
template <> struct real_of<float2> { using type = float; };

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc += a*b
template <typename C> __host__ __device__ __forceinline__ void cfma(C &acc, C a, C b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a*b
template <typename C> __host__ __device__ __forceinline__ void cfms(C &acc, C a, C b) {
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}
// a / b (Smith's algorithm, avoids overflow in |b|^2)
template <typename C> __host__ __device__ __forceinline__ C cdiv(C a, C b) {
    using R = typename real_of<C>::type;
    R ar = a.x, ai = a.y, br = b.x, bi = b.y;
    if (fabs(br) >= fabs(bi)) {
        R r = bi / br, d = br + bi * r;
        return mk((ar + ai * r) / d, (ai - ar * r) / d);
    } else {
        R r = br / bi, d = bi + br * r;
        return mk((ar * r + ai) / d, (ai * r - ar) / d);
    }
}
// Reciprocal 1/x: on the device the hardware approximation refined by Newton-Raphson
// (y <- y + y (1 - x y), one step for FP32, two for FP64, from the ~2^-20 seed of the
// FP64 approximation), within an ulp or so of the rounded quotient; plain division on
// the host.  Used on the pivot chain of the LU, where a full IEEE division sits on the
// critical path of every column step.
__host__ __device__ __forceinline__ float rcp_nr(float x) {
#ifdef __CUDA_ARCH__
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    const float e = fmaf(-x, y, 1.0f);
    return fmaf(y, e, y);
#else
    return 1.0f / x;
#endif
}
__host__ __device__ __forceinline__ double rcp_nr(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
#else
    return 1.0 / x;
#endif
}
// 1 / b with the components scaled by max(|re|, |im|) first (no over/underflow of |b|^2)
template <typename C> __host__ __device__ __forceinline__ C crecip(C b) {
    using R = typename real_of<C>::type;
    const R s = fmax(fabs(b.x), fabs(b.y));
    const R rs = rcp_nr(s);
    const R br = b.x * rs, bi = b.y * rs;
    const R d = rcp_nr(br * br + bi * bi);
    return mk(br * d * rs, -bi * d * rs);
}
template <typename C> __host__ __device__ __forceinline__ typename real_of<C>::type cabs1(C a) {
    return fabs(a.x) + fabs(a.y);
}
template <typename C> __host__ __device__ __forceinline__ C czero() { return mk((typename real_of<C>::type)0, (typename real_of<C>::type)0); }

__device__ __forceinline__ double2 to_c64(float2 a) { return make_double2((double)a.x, (double)a.y); }
__device__ __forceinline__ double2 to_c64(double2 a) { return a; }
__device__ __forceinline__ float2 to_c32(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ float2 to_c32(float2 a) { return a; }
template <typename C> __device__ __forceinline__ C conv(double2 a);
template <> __device__ __forceinline__ double2 conv<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 conv<float2>(double2 a) { return to_c32(a); }

// ---------------------------------------------------------------- error handling
void grim_set_error(const std::string &msg);
int grim_fail(int code, const std::string &msg);
int grim_cuda_check(cudaError_t e, const char *what);

#define GRIM_CHECK_CUDA(call)                                                     \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess) return grim_cuda_check(_e, #call);                 \
    } while (0)

// After every kernel launch: count it, check the launch, and (profiling on) record an
// end event so that consecutive events on the stream bracket each kernel.
#define GRIM_CHECK_LAUNCH_W(h, what, flops, bytes)                                \
    do {                                                                          \
        (h)->launches++;                                                          \
        cudaError_t _e = cudaGetLastError();                                      \
        if (_e != cudaSuccess) return grim_cuda_check(_e, what);                  \
        if ((h)->profiling) grim_prof_mark((h), (what), (double)(flops), (double)(bytes)); \
    } while (0)
#define GRIM_CHECK_LAUNCH(h, what) GRIM_CHECK_LAUNCH_W(h, what, 0.0, 0.0)

#define GRIM_TRY(call)                                                            \
    do {                                                                          \
        int _s = (call);                                                          \
        if (_s != GRIM_OK) return _s;                                             \
    } while (0)

// ---------------------------------------------------------------- context
struct grim_context {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    // named, grow-only device workspace buffers (stream-ordered allocations)
    std::unordered_map<std::string, std::pair<void *, size_t>> ws;
    grim_solve_info last{};
    int sm_count = 148;
    // error flag of the tensor-core kernels (device int, zeroed at first use)
    int *tc_err = nullptr;
    // factorization look-ahead: a high-priority stream for the panel chain, a low-priority
    // one for the wide trailing updates, and the events that order them (created lazily)
    cudaStream_t chain = nullptr, bulk = nullptr;
    std::vector<cudaEvent_t> events;
    // tile-shape overrides set by the autotuner (0 = built-in rule)
    int tune_solve_bn = 0;  // output-tile width of the right-hand-side GEMMs (64 or 128)
    int tune_gs_block = 0;  // row block of the packed-panel solve (256 or 512)
    // pivoting of later factorizations (GRIM_PIVOT_*): certified diagonal pivots with the
    // partial-pivoting fallback, static diagonal pivots, or partial pivoting throughout;
    // set per call by the solves that take a pivot mode, and by grim_set_tuning
    int pivot_mode = 0;
    // grouped factorization: the instantiated CUDA graph of the last plan, the key it was
    // captured for (element size, orders, device buffers it reads) and its launch count
    cudaGraphExec_t grp_exec = nullptr;
    std::vector<int64_t> grp_key;
    int64_t grp_graph_launches = 0;
    // profiling: one event per launch (plus a start event), aggregated by kernel name
    int profiling = 0;
    cudaEvent_t prof_start = nullptr;
    struct ProfMark {
        std::string name;
        cudaEvent_t ev;
        double flops, bytes;
    };
    std::vector<ProfMark> marks;
};

void grim_prof_mark(grim_context *h, const char *name, double flops, double bytes);

// Ensure a named workspace of at least `bytes` exists; returns its pointer in *out.
int grim_workspace(grim_context *h, const char *name, size_t bytes, void **out);

// Gauss-Legendre rules in constant memory, filled at context creation.
// Orders 1..GRIM_MAX_GAUSS are stored at offset order*(order-1)/2.
#define GRIM_MAX_GAUSS 32
int grim_upload_gauss(void);

// Scoped device guard
// A kernel's dynamic shared-memory opt-in (cudaFuncSetAttribute) is a setting of the
// current device, so each call site remembers it per device, not per process.
#define GRIM_MAX_DEVICES 64
struct PerDeviceOnce {
    bool set[GRIM_MAX_DEVICES] = {};
    bool needed() const {
        int dev = -1;
        cudaGetDevice(&dev);
        return dev < 0 || dev >= GRIM_MAX_DEVICES || !set[dev];
    }
    void mark() {
        int dev = -1;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < GRIM_MAX_DEVICES) set[dev] = true;
    }
};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Event-timed region on the handle stream.
struct StreamTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit StreamTimer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    double stop_ms() {
        record();
        return elapsed_ms();
    }
    // record the end without waiting; elapsed_ms() reads the interval later
    void record() { cudaEventRecord(b, s); }
    double elapsed_ms() {
        float ms = 0.f;
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        return (double)ms;
    }
    ~StreamTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

static inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
